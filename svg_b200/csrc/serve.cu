// Serving loop: resident SVGs, continuous batching of SSSD / MSAD requests,
// builds admitted under a device-memory budget (with eviction and rebuild).
//
// No counterpart in the reference, which answers one query at a time on the
// host (SVG::SolveSSSD / SolveMSAD, SVG.cu:241-413, called from the
// interactive loops of kernel.cu).
//
// Threads: callers submit requests (any thread); a worker thread forms
// batches and launches them; a builder thread runs builds.  Device side: a
// pool of "lanes", each a CUDA stream with fixed pinned-host and device
// staging buffers and one query context per resident graph.  A batch is the
// oldest queued request (SSSD before MSAD unless an MSAD has waited long)
// plus the next queued requests of the same kind and graph that fit the lane's
// staging, taken from that graph's own queue; requests that arrive while batches
// run are admitted as soon as a lane frees up, and batches on different lanes
// (and a build on the library stream) overlap on the GPU.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <list>
#include <mutex>
#include <thread>
#include <unordered_map>

#include "engine.h"
#include "svg_b200.h"

namespace svgb {
namespace {

double now_s() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

enum ReqKind { kSSSD = 0, kMSAD = 1, kBuild = 2 };

constexpr double kMsadAgeLimit = 0.5;  // s an MSAD may wait while SSSD requests go first
constexpr int kCopiers = 4;

struct Request {
    int64_t ticket = 0;
    int kind = kSSSD;
    int graph = -1;
    int32_t s = 0, t = 0;
    std::vector<int32_t> srcs;
    std::vector<double> w;
    double t_submit = 0.0, t_done = 0.0;
    int status = SVG_OK;
    std::string error;
    double dist = 0.0;
    int32_t nres = 0;                 // MSAD: vertices in the result
    std::vector<double> dists;        // MSAD result, unless the caller gave buffers
    std::vector<int32_t> src_ids;
    int64_t edges = 0;                // build: SVG edges
    double build_ms = 0.0;            // build: device time
    bool into = false;                // MSAD result goes to the caller's buffers (either may be null)
    double* out_d = nullptr;
    int32_t* out_s = nullptr;
};

struct GraphEntry {
    svg_mesh* mesh = nullptr;
    svg_build_opts opts{};
    svg_graph* g = nullptr;  // null while evicted or building
    bool building = false;
    bool owned = true;       // built by the server (freed on eviction)
    int inflight = 0;        // batches using it
    double last_used = 0.0;
    int64_t bytes = 0;
    int64_t build_ticket = 0;
    std::deque<Request*> waiting;  // queries held while (re)building
    std::deque<Request*> q[2];     // queued queries of this graph by kind, oldest first
};

struct Lane {
    cudaStream_t st = nullptr;
    cudaEvent_t ev = nullptr;
    bool busy = false;
    bool draining = false;            // results being copied out (worker, unlocked)
    int kind = 0, graph = -1, nv = 0;
    std::vector<Request*> batch;
    // staging: host pinned and device, fixed at creation
    char* h_in = nullptr;
    char* h_out = nullptr;
    char* d_in = nullptr;
    char* d_out = nullptr;
    size_t in_bytes = 0, out_bytes = 0;
    std::unordered_map<int, svg_qctx*> ctx;
    double t_launch = 0.0;
};

}  // namespace
}  // namespace svgb

using namespace svgb;

struct svg_server {
    svg_server_opts o{};
    std::mutex mu;
    std::condition_variable cv_work, cv_build, cv_done;
    // queued queries: per graph and kind (GraphEntry::q), the oldest-first
    // order of each kind as tickets (entries no longer in `queued` are skipped),
    // and the ticket -> request map of everything queued
    std::deque<int64_t> fifo[2];
    std::unordered_map<int64_t, Request*> queued;
    std::deque<Request*> builds;                  // build requests (graph index in Request::graph)
    std::unordered_map<int64_t, Request*> done;
    std::deque<GraphEntry> graphs;                // deque: entries stay put while the builder runs unlocked
    std::vector<Lane> lanes;
    std::thread worker, builder;
    std::vector<std::thread> copiers;             // copy finished batches out of pinned staging
    std::deque<Lane*> copy_q;
    std::condition_variable cv_copy;
    bool stop = false;
    int64_t next_ticket = 1;
    int64_t resident_bytes = 0;
    // counters
    int64_t batches = 0, batched_requests = 0, evictions = 0, rebuilds = 0;
    int dev = 0;
    int cluster = 0;  // blocks per query (0: one block)
    int slots = 1;    // queries a lane serves at once
    int sms = 0;
};

namespace {

int64_t graph_bytes(const svg_graph* g) {
    const int64_t V = g->nv, E = g->nnz;
    return 8 * (V + 1) + 4 * E + 8 * E + (g->with_paths ? 24 * E : 0) + 12 * V;
}

int64_t ctx_bytes_nv(int64_t V, int slots) {
    return (int64_t)slots * (8 * V + 16 * V + 16 * V + 8 * (2 * V + 64) + 4 * V + 2048);
}

int64_t ctx_bytes(const svg_graph* g, int slots) { return ctx_bytes_nv(g->nv, slots); }

void finish_request(svg_server* S, Request* r, int status, const std::string& err) {
    r->status = status;
    r->error = err;
    r->t_done = now_s();
    S->done[r->ticket] = r;
}

// Queue a query of a resident graph.  Called with S->mu held.
void enqueue(svg_server* S, Request* r) {
    S->graphs[(size_t)r->graph].q[r->kind].push_back(r);
    S->fifo[r->kind].push_back(r->ticket);
    S->queued[r->ticket] = r;
}

// Oldest queued request of a kind (nullptr if none).  Called with S->mu held.
Request* oldest(svg_server* S, int kind) {
    auto& f = S->fifo[kind];
    while (!f.empty()) {
        auto it = S->queued.find(f.front());
        if (it != S->queued.end()) return it->second;
        f.pop_front();
    }
    return nullptr;
}

bool graph_has_queued(const GraphEntry& G) { return !G.q[0].empty() || !G.q[1].empty(); }

// Launch a batch on a free lane.  Called with S->mu held.
void launch_batch(svg_server* S, Lane& L) {
    // short requests first: the oldest SSSD, unless the oldest MSAD is older
    // than it and has waited past the age limit (MSAD cannot starve)
    Request* so = oldest(S, kSSSD);
    Request* mo = oldest(S, kMSAD);
    if (!so && !mo) return;
    Request* first = so ? so : mo;
    if (so && mo && mo->t_submit < so->t_submit && now_s() - mo->t_submit >= kMsadAgeLimit) first = mo;
    const int kind = first->kind, gi = first->graph;
    GraphEntry& G = S->graphs[(size_t)gi];
    const int V = G.g->nv;
    // gather the batch: oldest first, same kind and graph, within staging capacity
    std::vector<Request*> batch;
    size_t in_used = 0, out_used = 0, nsrc = 0;
    const size_t max_n = (size_t)(kind == kSSSD ? S->o.max_batch : S->o.max_batch_msad);
    auto& gq = G.q[kind];  // this graph's queue of the kind: `first` is at its front
    while (!gq.empty() && batch.size() < max_n) {
        Request* r = gq.front();
        size_t in_need, out_need;
        if (kind == kSSSD) {
            in_need = 8;
            out_need = 8;
        } else {
            in_need = 8 + r->srcs.size() * 12;
            out_need = (size_t)V * 12;
        }
        // 1 KiB slack covers the 256-byte alignment of the packed sections
        if (!batch.empty() && (in_used + in_need + 1024 > L.in_bytes || out_used + out_need + 1024 > L.out_bytes))
            break;
        gq.pop_front();
        S->queued.erase(r->ticket);
        if (batch.empty() && (in_need + 1024 > L.in_bytes || out_need + 1024 > L.out_bytes)) {
            finish_request(S, r, SVG_ERR_ARG, "request larger than the serving lane's staging buffers");
            continue;
        }
        in_used += in_need;
        out_used += out_need;
        nsrc += r->srcs.size();
        batch.push_back(r);
    }
    if (batch.empty()) return;
    L.batch = batch;  // owned by the lane from here on (reported failed if a launch step throws)
    // per-lane context for this graph
    svg_qctx*& ctx = L.ctx[gi];
    if (!ctx) ctx = qctx_create(G.g, S->slots, L.st, S->cluster);
    const int n = (int)batch.size();
    auto al = [](size_t x) { return (x + 255) / 256 * 256; };
    if (kind == kSSSD) {
        int32_t* hs = reinterpret_cast<int32_t*>(L.h_in);
        int32_t* ht = hs + n;
        for (int i = 0; i < n; ++i) {
            hs[i] = batch[(size_t)i]->s;
            ht[i] = batch[(size_t)i]->t;
        }
        SVG_CUDA(cudaMemcpyAsync(L.d_in, L.h_in, 8 * (size_t)n, cudaMemcpyHostToDevice, L.st));
        int32_t* ds = reinterpret_cast<int32_t*>(L.d_in);
        qctx_sssd(ctx, n, ds, ds + n, reinterpret_cast<double*>(L.d_out), L.st);
        SVG_CUDA(cudaMemcpyAsync(L.h_out, L.d_out, 8 * (size_t)n, cudaMemcpyDeviceToHost, L.st));
    } else {
        const size_t o_off = 0, o_src = al(8 * ((size_t)n + 1)), o_w = o_src + al(4 * std::max<size_t>(nsrc, 1));
        int64_t* hoff = reinterpret_cast<int64_t*>(L.h_in + o_off);
        int32_t* hsrc = reinterpret_cast<int32_t*>(L.h_in + o_src);
        double* hw = reinterpret_cast<double*>(L.h_in + o_w);
        size_t k = 0;
        hoff[0] = 0;
        for (int i = 0; i < n; ++i) {
            const Request* r = batch[(size_t)i];
            for (size_t j = 0; j < r->srcs.size(); ++j, ++k) {
                hsrc[k] = r->srcs[j];
                hw[k] = r->w[j];
            }
            hoff[i + 1] = (int64_t)k;
        }
        const size_t in_total = o_w + 8 * std::max<size_t>(nsrc, 1);
        SVG_CUDA(cudaMemcpyAsync(L.d_in, L.h_in, in_total, cudaMemcpyHostToDevice, L.st));
        double* dd = reinterpret_cast<double*>(L.d_out);
        int32_t* di = reinterpret_cast<int32_t*>(L.d_out + al(8 * (size_t)n * V));
        qctx_msad(ctx, n, reinterpret_cast<int64_t*>(L.d_in + o_off), reinterpret_cast<int32_t*>(L.d_in + o_src),
                  reinterpret_cast<double*>(L.d_in + o_w), dd, di, L.st);
        SVG_CUDA(cudaMemcpyAsync(L.h_out, L.d_out, al(8 * (size_t)n * V) + 4 * (size_t)n * V, cudaMemcpyDeviceToHost,
                                 L.st));
    }
    SVG_CUDA(cudaEventRecord(L.ev, L.st));
    L.busy = true;
    L.kind = kind;
    L.graph = gi;
    L.nv = V;
    L.t_launch = now_s();
    G.inflight += 1;
    G.last_used = L.t_launch;
    S->batches += 1;
    S->batched_requests += n;
}

// Copy a finished batch's results out of the lane's pinned staging into the
// requests.  Runs without the lock: the lane is busy and its requests are in
// neither the queues nor `done`, so no other thread touches them.
void copy_results(Lane& L) {
    const int n = (int)L.batch.size();
    if (L.kind == kSSSD) {
        const double* ho = reinterpret_cast<const double*>(L.h_out);
        for (int i = 0; i < n; ++i) {
            Request* r = L.batch[(size_t)i];
            r->dist = ho[i];
            r->status = ho[i] < 0.0 ? SVG_ERR_STATE : SVG_OK;
        }
        return;
    }
    const size_t V = (size_t)L.nv;
    const size_t ob = (8 * (size_t)n * V + 255) / 256 * 256;
    const double* hd = reinterpret_cast<const double*>(L.h_out);
    const int32_t* hi = reinterpret_cast<const int32_t*>(L.h_out + ob);
    for (int i = 0; i < n; ++i) {
        Request* r = L.batch[(size_t)i];
        const double* d = hd + (size_t)i * V;
        const int32_t* si = hi + (size_t)i * V;
        if (r->into) {
            if (r->out_d) std::memcpy(r->out_d, d, 8 * V);
            if (r->out_s) std::memcpy(r->out_s, si, 4 * V);
        } else {
            r->dists.assign(d, d + V);
            r->src_ids.assign(si, si + V);
        }
        r->nres = (int32_t)V;
        r->status = SVG_OK;
    }
}

// Publish a batch whose results were copied.  Called with S->mu held.
void publish_batch(svg_server* S, Lane& L) {
    const double t = now_s();
    for (Request* r : L.batch) {
        r->t_done = t;
        S->done[r->ticket] = r;
    }
    S->graphs[(size_t)L.graph].inflight -= 1;
    L.batch.clear();
    L.busy = false;
    L.draining = false;
}

// launch_batch with its failures reported on the batch's requests.  Called
// with S->mu held; true if a batch was launched.
bool launch_guarded(svg_server* S, Lane& L) {
    try {
        launch_batch(S, L);
        return L.busy;
    } catch (const SvgError& e) {
        // the batch's requests were taken off the queues: report them failed
        for (Request* r : L.batch) finish_request(S, r, e.code, e.msg);
    } catch (const CudaFail& e) {
        cudaGetLastError();
        for (Request* r : L.batch) finish_request(S, r, SVG_ERR_CUDA, e.where);
    }
    L.batch.clear();
    L.busy = false;
    return false;
}

void worker_main(svg_server* S) {
    cudaSetDevice(S->dev);
    std::unique_lock<std::mutex> lk(S->mu);
    while (!S->stop) {
        bool progressed = false;
        std::vector<Lane*> ready;
        for (auto& L : S->lanes)
            if (L.busy && !L.draining && cudaEventQuery(L.ev) == cudaSuccess) {
                L.draining = true;
                ready.push_back(&L);
            }
        if (!ready.empty()) {
            for (Lane* L : ready) S->copy_q.push_back(L);
            S->cv_copy.notify_all();
            progressed = true;
        }
        for (auto& L : S->lanes) {
            if (L.busy || S->queued.empty()) continue;
            progressed |= launch_guarded(S, L);
        }
        bool any_busy = false;
        for (auto& L : S->lanes) any_busy |= L.busy;
        if (!progressed) {
            if (any_busy)
                S->cv_work.wait_for(lk, std::chrono::microseconds(20));
            else
                S->cv_work.wait_for(lk, std::chrono::milliseconds(5));
        }
    }
}

// Copier threads: results of finished batches leave the lane's pinned
// staging here, off the worker thread, which keeps launching meanwhile.
void copier_main(svg_server* S) {
    std::unique_lock<std::mutex> lk(S->mu);
    while (!S->stop) {
        if (S->copy_q.empty()) {
            S->cv_copy.wait_for(lk, std::chrono::milliseconds(5));
            continue;
        }
        Lane* L = S->copy_q.front();
        S->copy_q.pop_front();
        lk.unlock();
        copy_results(*L);
        lk.lock();
        publish_batch(S, *L);
        S->cv_done.notify_all();
        S->cv_work.notify_all();
    }
}

// Free least-recently-used idle graphs until `need` more bytes fit.
bool make_room(svg_server* S, int64_t need, int keep) {
    while (S->resident_bytes + need > S->o.hbm_budget) {
        int victim = -1;
        for (size_t i = 0; i < S->graphs.size(); ++i) {
            GraphEntry& G = S->graphs[i];
            if ((int)i == keep || !G.g || G.inflight > 0 || !G.owned) continue;
            if (graph_has_queued(G)) continue;
            if (victim < 0 || G.last_used < S->graphs[(size_t)victim].last_used) victim = (int)i;
        }
        if (victim < 0) return false;
        GraphEntry& G = S->graphs[(size_t)victim];
        for (auto& L : S->lanes) {
            auto it = L.ctx.find(victim);
            if (it != L.ctx.end()) {
                qctx_free(it->second);
                L.ctx.erase(it);
            }
        }
        svg_graph_free(G.g);
        G.g = nullptr;
        S->resident_bytes -= G.bytes;
        G.bytes = 0;
        S->evictions += 1;
    }
    return true;
}

// Work a graph needs once before queries, done unlocked on the library stream
// so that the worker never waits on it while holding the lock: its bucket
// width and one query context per lane.
svg_status prepare_graph(svg_server* S, svg_graph* g, std::string& err, std::vector<svg_qctx*>& ctxs) {
    try {
        graph_delta(g, lib_stream());
        for (size_t i = 0; i < S->lanes.size(); ++i) ctxs.push_back(qctx_create(g, S->slots, lib_stream(), S->cluster));
    } catch (const SvgError& e) {
        err = e.msg;
        for (svg_qctx* c : ctxs) qctx_free(c);
        ctxs.clear();
        return e.code;
    } catch (const CudaFail& e) {
        cudaGetLastError();
        err = std::string("CUDA error ") + cudaGetErrorString(e.err) + " in " + e.where;
        for (svg_qctx* c : ctxs) qctx_free(c);
        ctxs.clear();
        return SVG_ERR_CUDA;
    }
    return SVG_OK;
}

// Hand the prepared contexts to the lanes.  Called with S->mu held.
void attach_contexts(svg_server* S, int gi, std::vector<svg_qctx*>& ctxs) {
    for (size_t i = 0; i < ctxs.size() && i < S->lanes.size(); ++i) {
        svg_qctx*& slot = S->lanes[i].ctx[gi];
        if (slot) qctx_free(slot);
        slot = ctxs[i];
    }
    ctxs.clear();
}

void builder_main(svg_server* S) {
    cudaSetDevice(S->dev);
    std::unique_lock<std::mutex> lk(S->mu);
    while (!S->stop) {
        if (S->builds.empty()) {
            S->cv_build.wait_for(lk, std::chrono::milliseconds(5));
            continue;
        }
        Request* r = S->builds.front();
        S->builds.pop_front();
        const int gi = r->graph;
        GraphEntry& G = S->graphs[(size_t)gi];
        // admission: the graph's estimated size plus the build's scratch
        svg_build_opts o = G.opts;
        const int64_t est_graph = (int64_t)G.mesh->h.nv * ((int64_t)o.K + 8) * (o.with_paths ? 36 : 12);
        const int64_t est_ctx = (int64_t)S->lanes.size() * ctx_bytes_nv(G.mesh->h.nv, S->slots);
        const int64_t scratch = std::max<int64_t>(S->o.hbm_budget / 4, (int64_t)64 << 20);
        if (!make_room(S, est_graph + est_ctx + scratch, gi)) {
            // graphs still in use may become evictable: wait for their queries to
            // drain and retry; with none in use the budget cannot hold this build
            bool busy = false;
            for (size_t i = 0; i < S->graphs.size(); ++i) {
                const GraphEntry& H = S->graphs[i];
                if ((int)i == gi || !H.g || !H.owned) continue;
                busy |= H.inflight > 0 || graph_has_queued(H);
            }
            if (busy) {
                S->builds.push_front(r);
                S->cv_build.wait_for(lk, std::chrono::milliseconds(2));
                continue;
            }
            G.building = false;
            const std::string err = "server HBM budget too small for this build";
            for (Request* q : G.waiting) finish_request(S, q, SVG_ERR_NOMEM, err);
            G.waiting.clear();
            finish_request(S, r, SVG_ERR_NOMEM, err);
            S->cv_done.notify_all();
            continue;
        }
        o.hbm_budget = std::max<int64_t>(S->o.hbm_budget - S->resident_bytes - est_graph - est_ctx, scratch);
        // no K/10 probe build on the serving GPU: a graph's first build runs in
        // vertex order, its rebuilds heaviest first by the costs the mesh
        // recorded.  Measured on the mixed workload (2 builds/s beside 2,000
        // queries/s): with the probe, builds p50 / p99 167 ms / 1.9 s and MSAD
        // p99 556 ms; without it 90 ms / 0.87 s and 56 ms.
        if (o.heavy_first == 2) o.heavy_first = 1;
        if (o.blocks <= 0 && S->o.build_blocks_per_sm > 0) o.blocks = S->sms * S->o.build_blocks_per_sm;
        svg_graph* g = nullptr;
        lk.unlock();
        svg_status st = svg_build(G.mesh, &o, &g);
        std::string err = st == SVG_OK ? "" : svg_last_error();
        if (st == SVG_OK) {
            svg_build_stats bs{};
            if (svg_graph_stats(g, &bs) == SVG_OK) {
                r->edges = bs.edges;
                r->build_ms = bs.ms_total;
            }
        }
        std::vector<svg_qctx*> ctxs;
        if (st == SVG_OK) {
            st = prepare_graph(S, g, err, ctxs);
            if (st != SVG_OK) svg_graph_free(g);
        }
        lk.lock();
        G.building = false;
        if (st == SVG_OK) {
            attach_contexts(S, gi, ctxs);
            G.g = g;
            G.bytes = graph_bytes(g) + (int64_t)S->lanes.size() * ctx_bytes(g, S->slots);
            S->resident_bytes += G.bytes;
            G.last_used = now_s();
            for (Request* q : G.waiting) enqueue(S, q);
            G.waiting.clear();
            S->cv_work.notify_all();
        } else {
            for (Request* q : G.waiting) finish_request(S, q, st, err);
            G.waiting.clear();
        }
        finish_request(S, r, st, err);
        S->cv_done.notify_all();
    }
}

}  // namespace

extern "C" {

void svg_server_opts_default(svg_server_opts* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->hbm_budget = (int64_t)40 << 30;
    o->lanes = 0;
    o->max_batch = 4;
    o->max_batch_msad = 1;
    o->build_blocks_per_sm = 1;
    o->slots_per_lane = 0;
    o->cluster = 0;
    o->staging_in_bytes = (int64_t)16 << 20;
    o->staging_out_bytes = (int64_t)64 << 20;
}

svg_status svg_server_create(const svg_server_opts* opts, svg_server** out) {
    if (!out) return SVG_ERR_ARG;
    *out = nullptr;
    svg_server* S = new svg_server();
    try {
        if (opts) S->o = *opts;
        else svg_server_opts_default(&S->o);
        if (S->o.lanes < 0 || S->o.max_batch < 1 || S->o.max_batch_msad < 1 || S->o.slots_per_lane < 0 ||
            S->o.staging_in_bytes < 4096 ||
            S->o.staging_out_bytes < 4096)
            throw SvgError{SVG_ERR_ARG, "bad server options"};
        SVG_CUDA(cudaGetDevice(&S->dev));
        SVG_CUDA(cudaDeviceGetAttribute(&S->sms, cudaDevAttrMultiProcessorCount, S->dev));
        if (S->o.build_blocks_per_sm < 0) throw SvgError{SVG_ERR_ARG, "build_blocks_per_sm must be >= 0"};
        int prio_lo = 0, prio_hi = 0;  // query lanes get the highest stream priority
        SVG_CUDA(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
        // kernel form and per-lane concurrency: the lanes share the GPU's resident queries
        // (blocks in the plain form, clusters otherwise); by default one lane per cluster
        int resident = 0;
        if (S->o.cluster < 0) {
            S->cluster = 0;
            resident = query_slots_per_sm() * S->sms;
        } else {
            if (S->o.cluster != 0 && S->o.cluster != 8 && S->o.cluster != 16)
                throw SvgError{SVG_ERR_ARG, "cluster must be 0, -1, 8 or 16"};
            S->cluster = S->o.cluster > 0 ? S->o.cluster : query_cluster_size();
            resident = query_cluster_slots(S->cluster);
        }
        if (S->o.lanes == 0) S->o.lanes = std::min(std::max(1, resident), 32);
        S->slots = S->o.slots_per_lane > 0 ? S->o.slots_per_lane : std::max(1, resident / S->o.lanes);
        S->lanes.resize((size_t)S->o.lanes);
        for (auto& L : S->lanes) {
            SVG_CUDA(cudaStreamCreateWithPriority(&L.st, cudaStreamNonBlocking, prio_hi));
            SVG_CUDA(cudaEventCreateWithFlags(&L.ev, cudaEventDisableTiming));
            L.in_bytes = (size_t)S->o.staging_in_bytes;
            L.out_bytes = (size_t)S->o.staging_out_bytes;
            SVG_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&L.h_in), L.in_bytes, cudaHostAllocDefault));
            SVG_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&L.h_out), L.out_bytes, cudaHostAllocDefault));
            L.d_in = static_cast<char*>(dev_alloc(L.in_bytes));
            L.d_out = static_cast<char*>(dev_alloc(L.out_bytes));
        }
        S->resident_bytes = (int64_t)S->lanes.size() * (S->o.staging_in_bytes + S->o.staging_out_bytes);
        S->worker = std::thread(worker_main, S);
        for (int i = 0; i < kCopiers; ++i) S->copiers.emplace_back(copier_main, S);
        S->builder = std::thread(builder_main, S);
    } catch (const SvgError& e) {
        set_error(e.msg);
        svg_server_free(S);
        return e.code;
    } catch (const CudaFail& e) {
        cudaGetLastError();
        set_error(std::string("CUDA error ") + cudaGetErrorString(e.err) + " in " + e.where);
        svg_server_free(S);
        return SVG_ERR_CUDA;
    }
    *out = S;
    return SVG_OK;
}

void svg_server_free(svg_server* S) {
    if (!S) return;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
    }
    S->cv_work.notify_all();
    S->cv_build.notify_all();
    S->cv_copy.notify_all();
    if (S->worker.joinable()) S->worker.join();
    for (auto& t : S->copiers)
        if (t.joinable()) t.join();
    if (S->builder.joinable()) S->builder.join();
    for (auto& L : S->lanes) {
        for (Request* r : L.batch) delete r;  // batches still on a lane at shutdown
        L.batch.clear();
        if (L.st) cudaStreamSynchronize(L.st);
        for (auto& kv : L.ctx) qctx_free(kv.second);
        if (L.h_in) cudaFreeHost(L.h_in);
        if (L.h_out) cudaFreeHost(L.h_out);
        dev_free(L.d_in);
        dev_free(L.d_out);
        if (L.ev) cudaEventDestroy(L.ev);
        if (L.st) cudaStreamDestroy(L.st);
    }
    for (auto& G : S->graphs)
        if (G.g && G.owned) svg_graph_free(G.g);
    for (auto& kv : S->queued) delete kv.second;  // fifo entries are tickets only
    for (Request* r : S->builds) delete r;
    for (auto& kv : S->done) delete kv.second;
    for (auto& G : S->graphs)
        for (Request* r : G.waiting) delete r;
    delete S;
}

svg_status svg_server_add_graph(svg_server* S, svg_graph* g, int32_t* graph_id) {
    if (!S || !g || !graph_id) {
        set_error("null argument");
        return SVG_ERR_ARG;
    }
    std::string err;
    std::vector<svg_qctx*> ctxs;
    svg_status pst = prepare_graph(S, g, err, ctxs);
    if (pst != SVG_OK) {
        set_error(err);
        return pst;
    }
    std::lock_guard<std::mutex> lk(S->mu);
    GraphEntry G;
    G.mesh = g->mesh;
    svg_build_opts_default(&G.opts);
    G.opts.K = g->K;
    G.g = g;
    G.owned = false;  // the caller's graph: never evicted, never freed by the server
    G.bytes = graph_bytes(g) + (int64_t)S->lanes.size() * ctx_bytes(g, S->slots);
    G.last_used = now_s();
    S->resident_bytes += G.bytes;
    S->graphs.push_back(std::move(G));
    *graph_id = (int32_t)S->graphs.size() - 1;
    attach_contexts(S, *graph_id, ctxs);
    return SVG_OK;
}

svg_status svg_server_submit_build(svg_server* S, svg_mesh* m, const svg_build_opts* opts, int32_t* graph_id,
                                   int64_t* ticket) {
    if (!S || !m || !opts || !graph_id || !ticket) {
        set_error("null argument");
        return SVG_ERR_ARG;
    }
    std::lock_guard<std::mutex> lk(S->mu);
    GraphEntry G;
    G.mesh = m;
    G.opts = *opts;
    G.building = true;
    S->graphs.push_back(std::move(G));
    const int gi = (int)S->graphs.size() - 1;
    Request* r = new Request();
    r->ticket = S->next_ticket++;
    r->kind = kBuild;
    r->graph = gi;
    r->t_submit = now_s();
    S->builds.push_back(r);
    *graph_id = gi;
    *ticket = r->ticket;
    S->cv_build.notify_all();
    return SVG_OK;
}

static svg_status submit_query(svg_server* S, Request* r) {
    std::lock_guard<std::mutex> lk(S->mu);
    if (r->graph < 0 || r->graph >= (int)S->graphs.size()) {
        delete r;
        set_error("unknown graph id");
        return SVG_ERR_ARG;
    }
    GraphEntry& G = S->graphs[(size_t)r->graph];
    r->ticket = S->next_ticket++;
    if (G.g) {
        const int V = G.g->nv;
        bool ok = r->kind == kSSSD ? (r->s >= 0 && r->s < V && r->t >= 0 && r->t < V) : true;
        for (int32_t v : r->srcs) ok &= v >= 0 && v < V;
        if (!ok) {
            finish_request(S, r, SVG_ERR_ARG, "vertex out of range");
            return SVG_OK;
        }
        enqueue(S, r);
        S->cv_work.notify_all();
    } else {
        // evicted or still building: hold it, and rebuild if nothing is building it
        G.waiting.push_back(r);
        if (!G.building) {
            G.building = true;
            Request* b = new Request();
            b->ticket = S->next_ticket++;
            b->kind = kBuild;
            b->graph = r->graph;
            b->t_submit = now_s();
            S->builds.push_back(b);
            S->rebuilds += 1;
            S->cv_build.notify_all();
        }
    }
    return SVG_OK;
}

svg_status svg_server_submit_sssd(svg_server* S, int32_t graph_id, int32_t s, int32_t t, int64_t* ticket) {
    if (!S || !ticket) return SVG_ERR_ARG;
    Request* r = new Request();
    r->kind = kSSSD;
    r->graph = graph_id;
    r->s = s;
    r->t = t;
    r->t_submit = now_s();
    svg_status st = submit_query(S, r);
    if (st == SVG_OK) *ticket = r->ticket;
    return st;
}

svg_status svg_server_submit_msad(svg_server* S, int32_t graph_id, int32_t n, const int32_t* srcs,
                                  const double* weights, int64_t* ticket) {
    if (!S || !ticket || n < 0 || (n > 0 && (!srcs || !weights))) return SVG_ERR_ARG;
    Request* r = new Request();
    r->kind = kMSAD;
    r->graph = graph_id;
    r->srcs.assign(srcs, srcs + n);
    r->w.assign(weights, weights + n);
    r->t_submit = now_s();
    svg_status st = submit_query(S, r);
    if (st == SVG_OK) *ticket = r->ticket;
    return st;
}

svg_status svg_server_submit_msad_into(svg_server* S, int32_t graph_id, int32_t n, const int32_t* srcs,
                                       const double* weights, double* dists, int32_t* src_ids, int64_t* ticket) {
    if (!S || !ticket || n < 0 || (n > 0 && (!srcs || !weights))) return SVG_ERR_ARG;
    Request* r = new Request();
    r->kind = kMSAD;
    r->graph = graph_id;
    r->srcs.assign(srcs, srcs + n);
    r->w.assign(weights, weights + n);
    r->into = true;
    r->out_d = dists;
    r->out_s = src_ids;
    r->t_submit = now_s();
    svg_status st = submit_query(S, r);
    if (st == SVG_OK) *ticket = r->ticket;
    return st;
}

svg_status svg_server_wait(svg_server* S, int64_t ticket, double timeout_s, svg_server_result* res) {
    if (!S || !res) return SVG_ERR_ARG;
    std::unique_lock<std::mutex> lk(S->mu);
    const double deadline = now_s() + timeout_s;
    while (S->done.find(ticket) == S->done.end()) {
        if (timeout_s >= 0 && now_s() >= deadline) {
            set_error("timeout");
            return SVG_ERR_STATE;
        }
        S->cv_done.wait_for(lk, std::chrono::milliseconds(1));
    }
    Request* r = S->done[ticket];
    res->ticket = r->ticket;
    res->status = r->status;
    res->kind = r->kind;
    res->graph_id = r->graph;
    res->latency_ms = (r->t_done - r->t_submit) * 1e3;
    res->dist = r->dist;
    res->n = r->nres;
    res->edges = r->edges;
    res->build_ms = r->build_ms;
    return SVG_OK;
}

svg_status svg_server_take(svg_server* S, int64_t ticket, double* dists, int32_t* src_ids) {
    if (!S) return SVG_ERR_ARG;
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->done.find(ticket);
    if (it == S->done.end()) {
        set_error("ticket not finished or unknown");
        return SVG_ERR_STATE;
    }
    Request* r = it->second;
    if (dists && !r->dists.empty()) std::memcpy(dists, r->dists.data(), sizeof(double) * r->dists.size());
    if (src_ids && !r->src_ids.empty()) std::memcpy(src_ids, r->src_ids.data(), sizeof(int32_t) * r->src_ids.size());
    S->done.erase(it);
    delete r;
    return SVG_OK;
}

svg_status svg_server_poll(svg_server* S, int32_t max, svg_server_result* res, int32_t* n_out) {
    if (!S || !n_out || (max > 0 && !res)) return SVG_ERR_ARG;
    std::lock_guard<std::mutex> lk(S->mu);
    int32_t n = 0;
    for (auto& kv : S->done) {
        if (n >= max) break;
        Request* r = kv.second;
        svg_server_result& x = res[n++];
        x.ticket = r->ticket;
        x.status = r->status;
        x.kind = r->kind;
        x.graph_id = r->graph;
        x.latency_ms = (r->t_done - r->t_submit) * 1e3;
        x.dist = r->dist;
        x.n = r->nres;
        x.edges = r->edges;
        x.build_ms = r->build_ms;
    }
    *n_out = n;
    return SVG_OK;
}

svg_status svg_server_resident(svg_server* S, int32_t max, int32_t* ids, int32_t* n_out) {
    if (!S || !n_out || (max > 0 && !ids)) return SVG_ERR_ARG;
    std::lock_guard<std::mutex> lk(S->mu);
    std::vector<std::pair<double, int32_t>> r;
    for (size_t i = 0; i < S->graphs.size(); ++i)
        if (S->graphs[i].g) r.emplace_back(-S->graphs[i].last_used, (int32_t)i);
    std::sort(r.begin(), r.end());
    int32_t n = 0;
    for (auto& x : r) {
        if (n >= max) break;
        ids[n++] = x.second;
    }
    *n_out = n;
    return SVG_OK;
}

svg_status svg_server_stats(svg_server* S, svg_server_stats_t* st) {
    if (!S || !st) return SVG_ERR_ARG;
    std::lock_guard<std::mutex> lk(S->mu);
    st->pending = (int64_t)S->queued.size();
    st->batches = S->batches;
    st->batched_requests = S->batched_requests;
    st->resident_bytes = S->resident_bytes;
    st->evictions = S->evictions;
    st->rebuilds = S->rebuilds;
    int64_t res = 0;
    for (auto& G : S->graphs) res += G.g ? 1 : 0;
    st->resident_graphs = res;
    return SVG_OK;
}

}  // extern "C"
