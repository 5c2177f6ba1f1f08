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
#include <climits>

#include <cooperative_groups.h>

#include "engine.h"

namespace svgb {

namespace {

#ifndef SVG_Q_THREADS
#define SVG_Q_THREADS 512
#endif
#ifndef SVG_Q_UNROLL
#define SVG_Q_UNROLL 4
#endif
constexpr int kQThreads = SVG_Q_THREADS;
// edges per lane whose loads are issued together before any is used: the
// gather of the head's distance waits on the adjacency load, so issuing
// several of these chains at once hides most of their latency
constexpr int kQUnroll = SVG_Q_UNROLL;
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
                    const int64_t e0 = P.off[u], e1 = P.off[u + 1];
                    for (int64_t eb = e0 + lane; eb < e1; eb += 32 * kQUnroll) {
                        int wv[kQUnroll];
                        double nd[kQUnroll];
#pragma unroll
                        for (int j = 0; j < kQUnroll; ++j) {
                            const int64_t e = eb + 32 * j;
                            wv[j] = e < e1 ? __ldg(&P.adj[e]) : -1;
                            nd[j] = e < e1 ? du + __ldg(&P.w[e]) : 0.0;
                        }
                        unsigned long long curd[kQUnroll];
                        long long curs[kQUnroll];
#pragma unroll
                        for (int j = 0; j < kQUnroll; ++j) {
                            curd[j] = kInfBits;
                            curs[j] = -1;
                            if (wv[j] < 0) continue;
                            if (kSSSD) {
                                curd[j] = S.dist[wv[j]];
                            } else {
                                DS z = S.ds[wv[j]];
                                curd[j] = z.d;
                                curs[j] = z.s;
                            }
                        }
#pragma unroll
                        for (int j = 0; j < kQUnroll; ++j) {
                            const int w = wv[j];
                            if (w < 0 || !(nd[j] < as_d(curd[j]))) continue;
                            bool improved = false, first = false;
                            if (kSSSD) {
                                unsigned long long old = atomicMin(&S.dist[w], as_b(nd[j]));
                                improved = nd[j] < as_d(old);
                                first = old == kInfBits;
                            } else {
                                DS cur;
                                cur.d = curd[j];
                                cur.s = curs[j];
                                while (nd[j] < as_d(cur.d)) {
                                    DS nw;
                                    nw.d = as_b(nd[j]);
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
                            double f = kSSSD ? nd[j] + hdist(P.pos, w, tgt) : nd[j];
                            if (f < thr) {
                                if (atomicExch(&S.nflag[w], xst) != xst) S.next[atomicAdd(&s_nextN, 1)] = w;
                            } else if (atomicExch(&S.fflag[w], fst2) != fst2) {
                                int k = atomicAdd(&s_farN, 1);
                                if (k < P.list_cap) S.far[k] = w;
                                else s_overflow = 1;
                            }
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

// ---------------------------------------------------------------------------
// Cluster form: one query per thread-block cluster (8 or 16 SMs).  A batch runs
// only as many queries at once as there are clusters, so each query's
// distance and flag arrays stay in L2 while many SMs expand its frontier;
// per-block query concurrency (the single-block form above) thrashes L2 on
// large graphs.  The search is the same near-far label-correcting one, with:
//   * cluster barriers (hardware, no spinning) in place of __syncthreads;
//   * the phase counters in the first block's shared memory, reached by the
//     others through distributed shared memory, appended to with one atomic
//     per warp; each counter is triple-buffered by phase number, so that the
//     first block resets the copy nobody reads or writes in this phase;
//   * every decision (leave a loop, move the threshold) taken from values
//     read after a barrier and not written again before the next one, so all
//     blocks of a cluster take the same branches and meet at every barrier;
//   * mutable per-query arrays read through L2 (ld.global.cg): other SMs
//     write them, and L1 is not coherent across SMs.

#ifndef SVG_QC_THREADS
#define SVG_QC_THREADS 512
#endif
#ifndef SVG_QC_MINB
#define SVG_QC_MINB 2  // two blocks per SM (64 registers): twice the warps to hide load latency
#endif
constexpr int kCThreads = SVG_QC_THREADS;

struct QCtl {
    unsigned long long fmin[3];  // smallest waiting priority, by threshold move
    int nearA[3];                // near list filled by the far split
    int farB[3];                 // far list filled by the split and the drain
    int nextX[3];                // next near list, by drain round
    int touch;                   // SSSD: vertices whose distance left +inf
    int q;                       // query being served
    int init_far;                // far list length after the sources
    uint32_t stamp;              // slot stamp at the query's start
};

// Append the lanes with pred set to a list whose length is *counter (which may
// live in another block's shared memory): one atomic per warp.  Every lane of
// the warp must call it.  Returns the lane's position, or -1.
__device__ __forceinline__ int warp_append(bool pred, int* counter, int lane) {
    const unsigned m = __ballot_sync(0xffffffffu, pred);
    if (m == 0) return -1;
    const int first = __ffs(m) - 1;
    int base = 0;
    if (lane == first) base = atomicAdd(counter, __popc(m));
    base = __shfl_sync(0xffffffffu, base, first);
    return pred ? base + __popc(m & ((1u << lane) - 1u)) : -1;
}

__device__ __forceinline__ unsigned long long warp_min_u64(unsigned long long x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long y = __shfl_xor_sync(0xffffffffu, x, o);
        x = y < x ? y : x;
    }
    return x;
}

__device__ __forceinline__ DS ld_ds(const DS* p) {
    const longlong2 z = __ldcg(reinterpret_cast<const longlong2*>(p));
    DS r;
    r.d = (unsigned long long)z.x;
    r.s = z.y;
    return r;
}

template <bool kSSSD, bool kSrc>
__global__ void __launch_bounds__(kCThreads, SVG_QC_MINB) k_query_cluster(QParams P) {
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    __shared__ QCtl s_ctl;
    QCtl* ctl = cl.map_shared_rank(&s_ctl, 0);
    const int csize = (int)cl.num_blocks();
    const int crank = (int)cl.block_rank();
    const int slot = (int)blockIdx.x / csize;
    Slot S = carve_slot(P, slot);
    const int tid = threadIdx.x, lane = tid & 31;
    const int nthr = csize * kCThreads, gtid = crank * kCThreads + tid;
    const int gwarp = gtid >> 5, nwarps = nthr >> 5;
    const bool leader = crank == 0 && tid == 0;
    const long long round_cap = 64LL * ((long long)P.nv + 16);

    for (;;) {
        if (leader) {
            ctl->q = atomicAdd(P.head, 1);
            ctl->stamp = P.slot_stamp[slot];
        }
        cl.sync();
        const int q = ctl->q;
        uint32_t stamp = ctl->stamp;
        cl.sync();  // q and stamp read everywhere before the leader moves on (or any block leaves)
        if (q >= P.n) break;
        const int tgt = kSSSD ? P.t[q] : -1;

        // ---------------- initialise
        if (leader) {
            for (int k = 0; k < 3; ++k) {
                ctl->fmin[k] = kInfBits;
                ctl->nearA[k] = 0;
                ctl->farB[k] = 0;
                ctl->nextX[k] = 0;
            }
            ctl->touch = 0;
        }
        if (!kSSSD) {
            for (int v = gtid; v < P.nv; v += nthr) {
                DS z;
                z.d = kInfBits;
                z.s = -1;
                S.ds[v] = z;
            }
        }
        cl.sync();
        stamp += 1;
        const uint32_t fst = stamp;
        if (leader) {
            int nf = 0;
            if (kSSSD) {
                const int s = P.s[q];
                S.dist[s] = as_b(0.0);
                S.touched[0] = s;
                ctl->touch = 1;
                S.far[nf++] = s;
                S.fflag[s] = fst;
            } else {
                // SVG.cu:358-364: assignments in listed order, the last weight of a repeated source wins
                const int64_t b = P.set_off[q], e = P.set_off[q + 1];
                for (int64_t i = b; i < e; ++i) {
                    DS z;
                    z.d = as_b(P.weights[i]);
                    z.s = P.srcs[i];
                    S.ds[P.srcs[i]] = z;
                }
                for (int64_t i = b; i < e; ++i) {
                    const int v = P.srcs[i];
                    if (S.fflag[v] != fst) {
                        S.fflag[v] = fst;
                        S.far[nf++] = v;
                    }
                }
            }
            ctl->init_far = nf;
        }
        cl.sync();
        int farN = ctl->init_far;
        int32_t *far = S.far, *far2 = S.far2, *near = S.near, *next = S.next;
        long long rounds = 0;
        int o = 0, gr = 0;
        bool over = false;

        // ---------------- main loop: move the threshold, drain near frontiers
        for (;;) {
            // the far counter keeps counting past the list's capacity, so an
            // overflow shows in the value every block reads after the barrier
            if (++rounds > round_cap || farN > P.list_cap) {
                over = true;
                break;
            }
            const int ob = o % 3;
            unsigned long long m = kInfBits;
            for (int i = gtid; i < farN; i += nthr) {
                const int v = __ldcg(&far[i]);
                const double d = kSSSD ? as_d(__ldcg(&S.dist[v])) : as_d(ld_ds(&S.ds[v]).d);
                const double f = kSSSD ? d + hdist(P.pos, v, tgt) : d;
                m = as_b(f) < m ? as_b(f) : m;
            }
            m = warp_min_u64(m);
            if (lane == 0 && m != kInfBits) atomicMin(&ctl->fmin[ob], m);
            if (leader) {
                const int nb = (o + 1) % 3;
                ctl->fmin[nb] = kInfBits;
                ctl->nearA[nb] = 0;
                ctl->farB[nb] = 0;
            }
            cl.sync();
            if (farN == 0) break;
            const double fmin = as_d(ctl->fmin[ob]);
            if (kSSSD && as_d(__ldcg(&S.dist[tgt])) <= fmin) break;  // no waiting path can beat the target
            const double thr = fmin + P.delta;
            stamp += 2;
            const uint32_t nst = stamp - 1, fst2 = stamp;
            // split far: below the threshold -> near, the rest -> far2 (deduplicated)
            for (int base = gwarp * 32; base < farN; base += nthr) {
                const int i = base + lane;
                bool to_near = false, to_far = false;
                int v = -1;
                if (i < farN) {
                    v = __ldcg(&far[i]);
                    const double d = kSSSD ? as_d(__ldcg(&S.dist[v])) : as_d(ld_ds(&S.ds[v]).d);
                    const double f = kSSSD ? d + hdist(P.pos, v, tgt) : d;
                    if (f < thr) to_near = atomicExch(&S.nflag[v], nst) != nst;
                    else to_far = atomicExch(&S.fflag[v], fst2) != fst2;
                }
                int p = warp_append(to_near, &ctl->nearA[ob], lane);
                if (p >= 0) near[p] = v;
                p = warp_append(to_far, &ctl->farB[ob], lane);
                if (p >= 0 && p < P.list_cap) far2[p] = v;
            }
            cl.sync();
            {
                int32_t* t = far; far = far2; far2 = t;
            }
            int nearN = ctl->nearA[ob];

            // drain the near frontier: one warp per vertex, lanes over its edges
            while (nearN > 0) {
                if (++rounds > round_cap) {
                    over = true;
                    break;
                }
                const int gb = gr % 3;
                stamp += 1;
                const uint32_t xst = stamp;
                if (leader) ctl->nextX[(gr + 1) % 3] = 0;
                for (int i = gwarp; i < nearN; i += nwarps) {
                    const int u = __ldcg(&near[i]);
                    double du;
                    long long su = 0;
                    if (kSSSD) {
                        du = as_d(__ldcg(&S.dist[u]));
                    } else {
                        const DS z = ld_ds(&S.ds[u]);
                        du = as_d(z.d);
                        su = z.s;
                    }
                    const int64_t e0 = __ldg(&P.off[u]), e1 = __ldg(&P.off[u + 1]);
                    for (int64_t eb = e0; eb < e1; eb += 32 * kQUnroll) {
                        int wv[kQUnroll];
                        double nd[kQUnroll];
#pragma unroll
                        for (int j = 0; j < kQUnroll; ++j) {
                            const int64_t e = eb + 32 * j + lane;
                            wv[j] = e < e1 ? __ldg(&P.adj[e]) : -1;
                            nd[j] = e < e1 ? du + __ldg(&P.w[e]) : 0.0;
                        }
                        unsigned long long curd[kQUnroll];
                        long long curs[kQUnroll];
#pragma unroll
                        for (int j = 0; j < kQUnroll; ++j) {
                            curd[j] = kInfBits;
                            curs[j] = -1;
                            if (wv[j] < 0) continue;
                            if (kSSSD) {
                                curd[j] = __ldcg(&S.dist[wv[j]]);
                            } else {
                                const DS z = ld_ds(&S.ds[wv[j]]);
                                curd[j] = z.d;
                                curs[j] = z.s;
                            }
                        }
#pragma unroll
                        for (int j = 0; j < kQUnroll; ++j) {
                            const int w = wv[j];
                            bool to_next = false, to_far = false, to_touch = false;
                            if (w >= 0 && nd[j] < as_d(curd[j])) {
                                bool improved = false;
                                if (kSSSD) {
                                    const unsigned long long old = atomicMin(&S.dist[w], as_b(nd[j]));
                                    improved = nd[j] < as_d(old);
                                    to_touch = old == kInfBits;
                                } else {
                                    DS cur;
                                    cur.d = curd[j];
                                    cur.s = curs[j];
                                    while (nd[j] < as_d(cur.d)) {
                                        DS nw;
                                        nw.d = as_b(nd[j]);
                                        nw.s = su;
                                        const DS prev = atomicCAS(&S.ds[w], cur, nw);
                                        if (prev.d == cur.d && prev.s == cur.s) {
                                            improved = true;
                                            break;
                                        }
                                        cur = prev;
                                    }
                                }
                                if (improved) {
                                    const double f = kSSSD ? nd[j] + hdist(P.pos, w, tgt) : nd[j];
                                    if (f < thr) to_next = atomicExch(&S.nflag[w], xst) != xst;
                                    else to_far = atomicExch(&S.fflag[w], fst2) != fst2;
                                }
                            }
                            int p;
                            if (kSSSD) {
                                p = warp_append(to_touch, &ctl->touch, lane);
                                if (p >= 0) S.touched[p] = w;
                            }
                            p = warp_append(to_next, &ctl->nextX[gb], lane);
                            if (p >= 0) next[p] = w;
                            p = warp_append(to_far, &ctl->farB[ob], lane);
                            if (p >= 0 && p < P.list_cap) far[p] = w;
                        }
                    }
                }
                cl.sync();
                nearN = ctl->nextX[gb];
                {
                    int32_t* t = near; near = next; next = t;
                }
                ++gr;
            }
            if (over) break;
            farN = ctl->farB[ob];
            ++o;
        }

        // ---------------- results (every block got here after the same barriers)
        const bool ovf = over;
        if (kSSSD) {
            if (leader) {
                const unsigned long long dt = __ldcg(&S.dist[tgt]);
                P.out[q] = ovf ? -1.0 : (dt == kInfBits ? DBL_MAX : as_d(dt));
            }
            cl.sync();  // the target's distance is read before the reset below
            const int tn = ctl->touch;
            for (int i = gtid; i < tn; i += nthr) S.dist[__ldcg(&S.touched[i])] = kInfBits;
        } else {
            double* od = P.out_dist + (size_t)q * P.nv;
            int32_t* os = kSrc ? P.out_src + (size_t)q * P.nv : nullptr;
            for (int v = gtid; v < P.nv; v += nthr) {
                const DS z = ld_ds(&S.ds[v]);
                od[v] = z.d == kInfBits ? DBL_MAX : (ovf ? -1.0 : as_d(z.d));
                if (kSrc) os[v] = (int32_t)z.s;
            }
        }
        if (leader) P.slot_stamp[slot] = stamp;
        cl.sync();
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

__global__ void k_fill_i32(int32_t* p, int64_t n, int32_t v) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = v;
}

// Parent pointers of n finished searches (SVG::GraphDistInfo::pathParentIndex,
// SVG.cu:396): parent[q*nv + v] = the smallest u with an edge u -> v such that
// dist[u] + w == dist[v] (the addition the searches relax with) and
// dist[u] < dist[v].  Every vertex a search reached except its sources has
// such an edge: the relaxation that left dist[v] final read some dist[u], and
// had dist[u] fallen after it, v would have been relaxed again.  The strict
// dist[u] < dist[v] keeps the pointers acyclic.  One warp per (query, row u);
// parent must hold INT_MAX on entry.
__global__ void k_parents(const int64_t* __restrict__ off, const int32_t* __restrict__ adj,
                          const double* __restrict__ w, int32_t nv, int32_t n, const double* __restrict__ dist,
                          int32_t* __restrict__ parent) {
    const int lane = threadIdx.x & 31;
    const int64_t rows = (int64_t)n * nv;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < rows; r += nw) {
        const int64_t q = r / nv;
        const int u = (int)(r - q * nv);
        const double* d = dist + q * nv;
        const double du = d[u];
        if (!(du < DBL_MAX)) continue;
        const int64_t e1 = __ldg(&off[u + 1]);
        for (int64_t e = __ldg(&off[u]) + lane; e < e1; e += 32) {
            const int v = __ldg(&adj[e]);
            const double dv = d[v];
            if (du < dv && du + __ldg(&w[e]) == dv) atomicMin(&parent[q * nv + v], u);
        }
    }
}

// INT_MAX (no parent edge) -> -1; a vertex that kept its own source label
// (src[v] == v) is a root, as the reference leaves a source's parent at -1.
__global__ void k_parents_finish(int32_t* parent, const int32_t* src, int32_t nv, int64_t total) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int v = (int)(i % nv);
        if (parent[i] == INT_MAX || (src && src[i] == v)) parent[i] = -1;
    }
}

}  // namespace

void query_parents(svg_graph* g, int32_t n, const double* d_dist, const int32_t* d_src, int32_t* d_parent,
                   cudaStream_t st) {
    if (n <= 0 || g->nv <= 0) return;
    const int64_t total = (int64_t)n * g->nv;
    k_fill_i32<<<256, 256, 0, st>>>(d_parent, total, INT_MAX);
    int dev = 0, sms = 0;
    SVG_CUDA(cudaGetDevice(&dev));
    SVG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int64_t want = (total + 7) / 8;  // blocks of 8 warps
    k_parents<<<(int)std::min<int64_t>(want, (int64_t)sms * 16), 256, 0, st>>>(g->off, g->adj, g->dist, g->nv, n,
                                                                               d_dist, d_parent);
    k_parents_finish<<<(int)std::min<int64_t>((total + 255) / 256, (int64_t)sms * 16), 256, 0, st>>>(
        d_parent, d_src, g->nv, total);
    SVG_CUDA(cudaGetLastError());
}

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

namespace {
#ifndef SVG_QC_CLUSTER
#define SVG_QC_CLUSTER 16
#endif

template <bool A, bool B>
cudaLaunchConfig_t cluster_config(cudaLaunchAttribute* at, int nclusters, int csize, cudaStream_t st) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)(nclusters * csize), 1, 1);
    cfg.blockDim = dim3(kCThreads, 1, 1);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    at->id = cudaLaunchAttributeClusterDimension;
    at->val.clusterDim.x = (unsigned)csize;
    at->val.clusterDim.y = 1;
    at->val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cfg;
}

void allow_large_clusters() {
    static bool done = false;
    if (done) return;
    SVG_CUDA(cudaFuncSetAttribute(k_query_cluster<true, false>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    SVG_CUDA(cudaFuncSetAttribute(k_query_cluster<false, true>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    SVG_CUDA(cudaFuncSetAttribute(k_query_cluster<false, false>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    done = true;
}

template <bool A, bool B>
void launch_cluster(const QParams& P, int nclusters, int csize, cudaStream_t st) {
    allow_large_clusters();
    cudaLaunchAttribute at;
    cudaLaunchConfig_t cfg = cluster_config<A, B>(&at, nclusters, csize, st);
    SVG_CUDA(cudaLaunchKernelEx(&cfg, k_query_cluster<A, B>, P));
}

int max_active_clusters(int csize) {
    allow_large_clusters();
    cudaLaunchAttribute at;
    cudaLaunchConfig_t cfg = cluster_config<false, true>(&at, 1, csize, nullptr);
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, k_query_cluster<false, true>, &cfg) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}
}  // namespace

// Blocks per query of the cluster form: 16 where such clusters can be
// scheduled, else 8 (portable).
int query_cluster_size() {
    static int cs = 0;
    if (cs == 0) cs = max_active_clusters(SVG_QC_CLUSTER) >= 1 ? SVG_QC_CLUSTER : 8;
    return cs;
}

// Clusters of `csize` blocks that the GPU runs at once.
int query_cluster_slots(int csize) {
    static int cached[17] = {0};
    if (csize < 1 || csize > 16) return 1;
    if (cached[csize] <= 0) cached[csize] = std::max(1, max_active_clusters(csize));
    return cached[csize];
}

namespace {
// Cluster size of one call: a context made with `adaptive` serves a batch that
// fits in the resident clusters of its size at that size (latency), and a
// larger batch with 8-block clusters, which pack the SMs more fully
// (throughput); otherwise the context's own size.
int call_cluster(const svg_qctx* c, int n) {
    if (!c->adaptive || c->cluster <= 8 || n <= query_cluster_slots(c->cluster)) return c->cluster;
    return 8;
}
}  // namespace

// Query blocks one SM holds at once (occupancy of the MSAD kernel, the larger one).
int query_slots_per_sm() {
    static int per_sm = 0;
    if (per_sm <= 0) {
        int b = 0;
        SVG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_query<false, true>, kQThreads, 0));
        per_sm = std::max(1, b);
    }
    return per_sm;
}

// Query scratch for `slots` concurrent queries of one graph: per slot the SSSD
// distances (kept at +inf between queries), the MSAD {dist, src} pairs, the
// stamp arrays and the frontier lists; one launch at a time may use it.
svg_qctx* qctx_create(svg_graph* g, int slots, cudaStream_t st, int cluster) {
    graph_delta(g, st);
    svg_qctx* c = new svg_qctx();
    c->g = g;
    c->slots = std::max(1, slots);
    c->cluster = std::max(0, cluster);
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
    if (c->cluster > 0) {
        const int cs = call_cluster(c, n);
        launch_cluster<true, false>(P, std::min(std::min(n, c->slots), query_cluster_slots(cs)), cs, st);
    } else
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
    const int nb = std::min(n, c->slots);
    if (c->cluster > 0) {
        const int cs = call_cluster(c, n);
        const int nc = std::min(nb, query_cluster_slots(cs));
        if (d_src_id) launch_cluster<false, true>(P, nc, cs, st);
        else launch_cluster<false, false>(P, nc, cs, st);
    } else if (d_src_id) {
        k_query<false, true><<<nb, kQThreads, 0, st>>>(P);
    } else {
        k_query<false, false><<<nb, kQThreads, 0, st>>>(P);
    }
    SVG_CUDA(cudaGetLastError());
}

namespace {
// The graph's own context for the synchronous batch entry points: as many
// clusters as run at once (cluster form), or every resident block (plain form).
svg_qctx* default_ctx(svg_graph* g) {
    if (!g->qdefault) {
        if (g->qform == SVG_QUERY_PLAIN) {
            int dev = 0, sms = 0;
            SVG_CUDA(cudaGetDevice(&dev));
            SVG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
            g->qdefault = qctx_create(g, query_slots_per_sm() * sms, lib_stream(), 0);
        } else {
            const int cs = query_cluster_size();
            g->qdefault = qctx_create(g, std::max(query_cluster_slots(cs), query_cluster_slots(8)), lib_stream(), cs);
            g->qdefault->adaptive = true;
        }
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
