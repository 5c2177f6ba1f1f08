// Batched shortest-path queries on the resident SVG (CSR).
//
// SVG::SolveSSSD / SolveMSAD (SVG.cu:241-251, 354-413) run a binary-heap A*
// (Euclidean heuristic) or Dijkstra on the host, one query at a time.  Here
// one thread block serves one query at a time, many blocks serve a batch,
// and each query is a near-far label-correcting search:
//   * a frontier ("near") of vertices whose distance improved and whose
//     priority f = dist (+ |p - p_t| for SSSD) is below a threshold is
//     relaxed in parallel, one warp per vertex, lanes over its edges;
//     distances fall by 64-bit atomicMin on the double's bit pattern
//     (non-negative doubles order like their bits), or, for MSAD with
//     source ids, by a 16-byte compare-and-swap of {dist, src};
//   * improved vertices above the threshold wait in a "far" list; when the
//     near frontier drains, the threshold moves to the smallest waiting
//     priority plus delta and those below it become the next frontier.
// The result is the exact shortest-path distance (label correcting).  SSSD
// stops once the target's distance is at most the threshold: with the
// reference's consistent heuristic no unsettled path can then be shorter.
// Per-slot stamp arrays replace clearing: a stamp is never reused.
#include <cfloat>

#include "engine.h"

namespace svgb {

namespace {

constexpr int kQThreads = 512;
constexpr unsigned long long kInfBits = 0x7FF0000000000000ull;  // +inf

struct alignas(16) DS {
    unsigned long long d;  // double bits
    long long s;           // source id (-1 = none)
};

struct QParams {
    const int64_t* off;
    const int32_t* adj;
    const double* w;
    const double* pos;     // 3*nv
    int32_t nv;
    int32_t n;             // queries
    double delta;
    // SSSD
    const int32_t* s;
    const int32_t* t;
    double* out;           // n
    // MSAD
    const int64_t* set_off;
    const int32_t* srcs;
    const double* weights;
    double* out_dist;      // n*nv
    int32_t* out_src;      // n*nv or null
    // scratch
    char* scratch;
    size_t slot_bytes;
    uint32_t* slot_stamp;  // per slot
    int32_t* head;
    int64_t list_cap;      // far list capacity (entries)
};

__device__ __forceinline__ double hdist(const double* pos, int a, int b) {
    double dx = pos[3 * a] - pos[3 * b], dy = pos[3 * a + 1] - pos[3 * b + 1], dz = pos[3 * a + 2] - pos[3 * b + 2];
    return sqrt(dx * dx + dy * dy + dz * dz);
}

__device__ __forceinline__ double as_d(unsigned long long b) { return __longlong_as_double((long long)b); }
__device__ __forceinline__ unsigned long long as_b(double d) { return (unsigned long long)__double_as_longlong(d); }

struct Slot {
    unsigned long long* dist;  // SSSD distances, nv, kept at +inf between queries
    DS* ds;                    // MSAD {dist, src}, nv, initialised per query
    uint32_t* nflag;           // nv
    uint32_t* fflag;           // nv
    int32_t* near;             // nv
    int32_t* next;             // nv
    int32_t* far;              // list_cap
    int32_t* far2;             // list_cap
    int32_t* touched;          // nv
};

__device__ Slot carve_slot(const QParams& P, int slot) {
    char* p = P.scratch + (size_t)slot * P.slot_bytes;
    size_t V = (size_t)P.nv;
    auto take = [&](size_t bytes) { char* q = p; p += (bytes + 255) / 256 * 256; return q; };
    Slot S;
    S.dist = reinterpret_cast<unsigned long long*>(take(8 * V));
    S.ds = reinterpret_cast<DS*>(take(16 * V));
    S.nflag = reinterpret_cast<uint32_t*>(take(4 * V));
    S.fflag = reinterpret_cast<uint32_t*>(take(4 * V));
    S.near = reinterpret_cast<int32_t*>(take(4 * V));
    S.next = reinterpret_cast<int32_t*>(take(4 * V));
    S.far = reinterpret_cast<int32_t*>(take(4 * (size_t)P.list_cap));
    S.far2 = reinterpret_cast<int32_t*>(take(4 * (size_t)P.list_cap));
    S.touched = reinterpret_cast<int32_t*>(take(4 * V));
    return S;
}

template <bool kSSSD, bool kSrc>
__global__ void __launch_bounds__(kQThreads) k_query(QParams P) {
    __shared__ int s_q;
    __shared__ int s_nearN, s_nextN, s_farN, s_far2N, s_touchN;
    __shared__ unsigned long long s_fmin;
    __shared__ uint32_t s_stamp;
    __shared__ int s_overflow;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = kQThreads / 32;
    Slot S = carve_slot(P, blockIdx.x);
    uint32_t* stamp_ctr = &P.slot_stamp[blockIdx.x];

    for (;;) {
        if (tid == 0) s_q = atomicAdd(P.head, 1);
        __syncthreads();
        const int q = s_q;
        if (q >= P.n) break;
        int tgt = -1;
        if (kSSSD) tgt = P.t[q];
        double thr;

        // ---------------- initialise
        if (tid == 0) {
            s_nearN = 0; s_farN = 0; s_touchN = 0; s_overflow = 0;
            s_stamp = *stamp_ctr + 1;
        }
        if (!kSSSD) {
            for (int v = tid; v < P.nv; v += kQThreads) {
                DS z;
                z.d = kInfBits;
                z.s = -1;
                S.ds[v] = z;
            }
        }
        __syncthreads();
        const uint32_t fst = s_stamp;  // far-list stamp of the first phase
        if (kSSSD) {
            int s = P.s[q];
            if (tid == 0) {
                S.dist[s] = as_b(0.0);
                S.touched[s_touchN++] = s;
                S.far[s_farN++] = s;
                S.fflag[s] = fst;
            }
        } else if (tid == 0) {
            // SVG.cu:358-364: assignments in listed order, the last weight of a repeated source wins
            int64_t b = P.set_off[q], e = P.set_off[q + 1];
            for (int64_t i = b; i < e; ++i) {
                DS z;
                z.d = as_b(P.weights[i]);
                z.s = P.srcs[i];
                S.ds[P.srcs[i]] = z;
            }
            for (int64_t i = b; i < e; ++i) {
                int v = P.srcs[i];
                if (S.fflag[v] != fst) {
                    S.fflag[v] = fst;
                    S.far[s_farN++] = v;
                }
            }
        }
        __syncthreads();
        thr = -1.0;
        // every loop below is bounded: a query that needs more rounds than this
        // reports -1 instead of spinning
        const long long round_cap = 64LL * ((long long)P.nv + 16);
        long long rounds = 0;

        // ---------------- main loop: move the threshold, drain near frontiers
        for (;;) {
            if (++rounds > round_cap) {
                if (tid == 0) s_overflow = 1;
                __syncthreads();
                break;
            }
            // smallest priority waiting in far
            if (tid == 0) s_fmin = kInfBits;
            __syncthreads();
            const int farN = s_farN;
            for (int i = tid; i < farN; i += kQThreads) {
                int v = S.far[i];
                double d = kSSSD ? as_d(S.dist[v]) : as_d(S.ds[v].d);
                double f = kSSSD ? d + hdist(P.pos, v, tgt) : d;
                atomicMin(&s_fmin, as_b(f));
            }
            __syncthreads();
            if (farN == 0) break;
            double fmin = as_d(s_fmin);
            if (kSSSD) {
                double dt = as_d(S.dist[tgt]);
                if (dt <= fmin) break;  // no waiting path can beat the target's distance
            }
            thr = fmin + P.delta;
            // split far: below the threshold -> near, the rest stays (deduplicated)
            if (tid == 0) { s_nearN = 0; s_far2N = 0; s_stamp += 2; }
            __syncthreads();
            const uint32_t nst = s_stamp - 1, fst2 = s_stamp;
            for (int i = tid; i < farN; i += kQThreads) {
                int v = S.far[i];
                double d = kSSSD ? as_d(S.dist[v]) : as_d(S.ds[v].d);
                double f = kSSSD ? d + hdist(P.pos, v, tgt) : d;
                if (f < thr) {
                    if (atomicExch(&S.nflag[v], nst) != nst) S.near[atomicAdd(&s_nearN, 1)] = v;
                } else if (atomicExch(&S.fflag[v], fst2) != fst2) {
                    S.far2[atomicAdd(&s_far2N, 1)] = v;
                }
            }
            __syncthreads();
            {
                int32_t* tmp = S.far; S.far = S.far2; S.far2 = tmp;
            }
            if (tid == 0) s_farN = s_far2N;
            __syncthreads();

            // drain the near frontier
            while (s_nearN > 0) {
                if (++rounds > round_cap) break;
                const int nearN = s_nearN;
                if (tid == 0) { s_nextN = 0; ++s_stamp; }
                __syncthreads();
                const uint32_t xst = s_stamp;
                for (int i = warp; i < nearN; i += nwarps) {
                    int u = S.near[i];
                    double du;
                    long long su = 0;
                    if (kSSSD) {
                        du = as_d(S.dist[u]);
                    } else {
                        DS z = S.ds[u];
                        du = as_d(z.d);
                        su = z.s;
                    }
                    int64_t e0 = P.off[u], e1 = P.off[u + 1];
                    for (int64_t e = e0 + lane; e < e1; e += 32) {
                        int w = P.adj[e];
                        double nd = du + P.w[e];
                        bool improved = false, first = false;
                        if (kSSSD) {
                            unsigned long long cur = S.dist[w];
                            if (nd < as_d(cur)) {
                                unsigned long long old = atomicMin(&S.dist[w], as_b(nd));
                                improved = nd < as_d(old);
                                first = old == kInfBits;
                            }
                        } else {
                            DS cur = S.ds[w];
                            while (nd < as_d(cur.d)) {
                                DS nw;
                                nw.d = as_b(nd);
                                nw.s = su;
                                DS prev = atomicCAS(&S.ds[w], cur, nw);
                                if (prev.d == cur.d && prev.s == cur.s) { improved = true; break; }
                                cur = prev;
                            }
                        }
                        if (!improved) continue;
                        if (kSSSD && first) {
                            int k = atomicAdd(&s_touchN, 1);
                            S.touched[k] = w;
                        }
                        double f = kSSSD ? nd + hdist(P.pos, w, tgt) : nd;
                        if (f < thr) {
                            if (atomicExch(&S.nflag[w], xst) != xst) S.next[atomicAdd(&s_nextN, 1)] = w;
                        } else if (atomicExch(&S.fflag[w], fst2) != fst2) {
                            int k = atomicAdd(&s_farN, 1);
                            if (k < P.list_cap) S.far[k] = w;
                            else s_overflow = 1;
                        }
                    }
                }
                __syncthreads();
                {
                    int32_t* tmp = S.near; S.near = S.next; S.next = tmp;
                }
                if (tid == 0) s_nearN = s_nextN;
                __syncthreads();
            }
            if (rounds > round_cap && tid == 0) s_overflow = 1;
            __syncthreads();
            if (s_overflow) break;
        }
        __syncthreads();

        // ---------------- results
        if (kSSSD) {
            if (tid == 0) {
                unsigned long long dt = S.dist[tgt];
                P.out[q] = s_overflow ? -1.0 : (dt == kInfBits ? DBL_MAX : as_d(dt));
            }
            __syncthreads();
            const int tn = s_touchN;
            for (int i = tid; i < tn; i += kQThreads) S.dist[S.touched[i]] = kInfBits;
        } else {
            double* od = P.out_dist + (size_t)q * P.nv;
            int32_t* os = kSrc ? P.out_src + (size_t)q * P.nv : nullptr;
            for (int v = tid; v < P.nv; v += kQThreads) {
                DS z = S.ds[v];
                od[v] = z.d == kInfBits ? DBL_MAX : (s_overflow ? -1.0 : as_d(z.d));
                if (kSrc) os[v] = (int32_t)z.s;
            }
        }
        if (tid == 0) *stamp_ctr = s_stamp;
        __syncthreads();
    }
}

__global__ void k_mean_weight(const double* w, int64_t n, double* out) {
    __shared__ double s[256];
    double acc = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        acc += w[i];
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int k = 128; k > 0; k >>= 1) {
        if ((int)threadIdx.x < k) s[threadIdx.x] += s[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(out, s[0]);
}

__global__ void k_fill(unsigned long long* p, size_t n, unsigned long long v) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        p[i] = v;
}

size_t al256(size_t x) { return (x + 255) / 256 * 256; }

}  // namespace

// Bucket width of the near-far search: the mean SVG edge length, computed once per graph.
double graph_delta(svg_graph* g, cudaStream_t st) {
    if (g->delta > 0.0) return g->delta;
    double* d_sum = dev_alloc_n<double>(1);
    SVG_CUDA(cudaMemsetAsync(d_sum, 0, sizeof(double), st));
    if (g->nnz > 0) k_mean_weight<<<256, 256, 0, st>>>(g->dist, g->nnz, d_sum);
    double sum = 0.0;
    SVG_CUDA(cudaMemcpyAsync(&sum, d_sum, sizeof(double), cudaMemcpyDeviceToHost, st));
    SVG_CUDA(cudaStreamSynchronize(st));
    dev_free(d_sum);
    double mean = g->nnz > 0 ? sum / (double)g->nnz : 1.0;
    g->delta = mean > 0.0 ? mean : 1.0;
    return g->delta;
}

// Query scratch for `slots` concurrent queries of one graph: per slot the SSSD
// distances (kept at +inf between queries), the MSAD {dist, src} pairs, the
// stamp arrays and the frontier lists; one launch at a time may use it.
svg_qctx* qctx_create(svg_graph* g, int slots, cudaStream_t st) {
    graph_delta(g, st);
    svg_qctx* c = new svg_qctx();
    c->g = g;
    c->slots = std::max(1, slots);
    const size_t V = (size_t)g->nv;
    c->list_cap = 2 * (int64_t)V + 64;
    c->slot_bytes = al256(8 * V) + al256(16 * V) + 4 * al256(4 * V) + 2 * al256(4 * (size_t)c->list_cap) + al256(4 * V);
    const size_t body = al256((size_t)c->slots * c->slot_bytes);
    const size_t need = body + al256(sizeof(uint32_t) * (size_t)c->slots) + 256;
    try {
        c->buf.reserve(need);
    } catch (...) {
        delete c;
        throw;
    }
    char* base = c->buf.as<char>();
    c->stamps = reinterpret_cast<uint32_t*>(base + body);
    c->head = reinterpret_cast<int32_t*>(base + body + al256(sizeof(uint32_t) * (size_t)c->slots));
    SVG_CUDA(cudaMemsetAsync(base, 0, need, st));  // stamps and flags start at 0
    for (int sl = 0; sl < c->slots; ++sl)          // SSSD distances start at +inf
        k_fill<<<64, 256, 0, st>>>(reinterpret_cast<unsigned long long*>(base + (size_t)sl * c->slot_bytes), V,
                                  kInfBits);
    SVG_CUDA(cudaGetLastError());
    SVG_CUDA(cudaStreamSynchronize(st));
    return c;
}

void qctx_free(svg_qctx* c) { delete c; }

namespace {
void fill_params(svg_qctx* c, QParams& P) {
    svg_graph* g = c->g;
    P.scratch = c->buf.as<char>();
    P.slot_bytes = c->slot_bytes;
    P.slot_stamp = c->stamps;
    P.head = c->head;
    P.list_cap = c->list_cap;
    P.off = g->off;
    P.adj = g->adj;
    P.w = g->dist;
    P.pos = g->mesh->d.pos;
    P.nv = g->nv;
    P.delta = g->delta;
}
}  // namespace

void qctx_sssd(svg_qctx* c, int32_t n, const int32_t* d_s, const int32_t* d_t, double* d_dist, cudaStream_t st) {
    if (n <= 0) return;
    QParams P{};
    fill_params(c, P);
    P.n = n;
    P.s = d_s;
    P.t = d_t;
    P.out = d_dist;
    SVG_CUDA(cudaMemsetAsync(P.head, 0, sizeof(int32_t), st));
    k_query<true, false><<<std::min(n, c->slots), kQThreads, 0, st>>>(P);
    SVG_CUDA(cudaGetLastError());
}

void qctx_msad(svg_qctx* c, int32_t n, const int64_t* d_off, const int32_t* d_src, const double* d_w, double* d_dist,
               int32_t* d_src_id, cudaStream_t st) {
    if (n <= 0) return;
    QParams P{};
    fill_params(c, P);
    P.n = n;
    P.set_off = d_off;
    P.srcs = d_src;
    P.weights = d_w;
    P.out_dist = d_dist;
    P.out_src = d_src_id;
    SVG_CUDA(cudaMemsetAsync(P.head, 0, sizeof(int32_t), st));
    if (d_src_id)
        k_query<false, true><<<std::min(n, c->slots), kQThreads, 0, st>>>(P);
    else
        k_query<false, false><<<std::min(n, c->slots), kQThreads, 0, st>>>(P);
    SVG_CUDA(cudaGetLastError());
}

namespace {
// The graph's own context for the synchronous batch entry points: two query
// blocks per SM.
svg_qctx* default_ctx(svg_graph* g) {
    if (!g->qdefault) {
        int dev = 0, sms = 0;
        SVG_CUDA(cudaGetDevice(&dev));
        SVG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        g->qdefault = qctx_create(g, 2 * sms, lib_stream());
    }
    return g->qdefault;
}

}  // namespace

svg_status run_sssd(svg_graph* g, int32_t n, const int32_t* d_s, const int32_t* d_t, double* d_dist) {
    if (n == 0) return SVG_OK;
    qctx_sssd(default_ctx(g), n, d_s, d_t, d_dist, lib_stream());
    return SVG_OK;
}

svg_status run_msad(svg_graph* g, int32_t n, const int64_t* d_off, const int32_t* d_src, const double* d_w,
                    double* d_dist, int32_t* d_src_id, int64_t total_srcs) {
    (void)total_srcs;
    if (n == 0) return SVG_OK;
    qctx_msad(default_ctx(g), n, d_off, d_src, d_w, d_dist, d_src_id, lib_stream());
    return SVG_OK;
}

}  // namespace svgb
