// SVG construction kernels and their host orchestration.
//
//  batched (the product path):
//    k_ich_batched  persistent: every lane pulls sources from a device work
//                   queue, runs one K-limited ICH, classifies the vertices it
//                   reached (direct = geodesic passes no vertex, decided from
//                   the first back-trace hop) and appends the direct ones to a
//                   candidate pool.  The loop is flat - one ICH step per
//                   iteration - so a lane that finishes takes new work at once
//                   instead of idling until its warp's slowest source ends.
//    exclusive scan of the per-source degrees -> CSR offsets
//    k_emit         one warp per source: bitonic-sort the candidates by vertex
//                   id in shared memory, keep the first K (the reference's
//                   ascending-j, cap-K rule, SVG.cu:44-75), trace their path
//                   ends in parallel, write the CSR row.
//  plain (the reference's form, for comparison):
//    k_ich_plain    one source per thread, grid-stride, full table reset per
//                   source and the O(V) emission scan of SVG.cu:44-75 with the
//                   full back-trace, into a V x K padded array; then
//                   k_compact packs it into the same CSR.
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cstring>

#include "engine.h"
#include "ich.cuh"

// Blocks of 128 lanes the batched kernel is compiled to fit per SM (register
// budget); 0 = no constraint.
#ifndef SVG_ICH_MIN_BLOCKS
#define SVG_ICH_MIN_BLOCKS 0
#endif
// The lane hash tables hold 2^shift times the slots of the base sizing below
// (fewer collisions, each a dependent round trip): vertex table
// SVG_TABLE_SHIFT, split table SVG_SPLIT_SHIFT.  Both at 1 measured 1.7-2 %
// faster at K = 500.
#ifndef SVG_TABLE_SHIFT
#define SVG_TABLE_SHIFT 1
#endif
#ifndef SVG_SPLIT_SHIFT
#define SVG_SPLIT_SHIFT SVG_TABLE_SHIFT
#endif
// 1: the path ends of the emitted rows are traced by a kernel of their own
// (k_trace, one thread per edge) after k_emit
#ifndef SVG_SPLIT_TRACE
#define SVG_SPLIT_TRACE 1
#endif
// blocks of 256 per SM k_trace is compiled to fit (register budget)
#ifndef SVG_TRACE_MIN_BLOCKS
#define SVG_TRACE_MIN_BLOCKS 4
#endif
// threads per block the batched kernel is compiled for (the launch may use fewer)
#ifndef SVG_ICH_TPB
#define SVG_ICH_TPB 128
#endif
#if SVG_ICH_MIN_BLOCKS > 0
#define SVG_ICH_BOUNDS __launch_bounds__(SVG_ICH_TPB, SVG_ICH_MIN_BLOCKS)
#else
#define SVG_ICH_BOUNDS __launch_bounds__(SVG_ICH_TPB)
#endif

namespace svgb {

struct PhaseOut {
    const int32_t* order;
    int32_t nsrc;
    int32_t* work;                 // work-queue head
    int32_t* retry;                // sources whose lane tables filled
    int32_t* retry_n;
    Cand* cand;
    unsigned long long* cand_used;
    int64_t cand_cap;
    int64_t* cand_start;           // per vertex
    int32_t* cand_n;
    int32_t* deg;
    int32_t* st_windows;
    int32_t* st_maxq;
    int32_t* st_flags;
    unsigned long long* acc;       // windows, generated, pseudo-sources, queue-drop sources
    // Cooperative warps: warp 0 of each of the first coop_warps blocks takes
    // the heaviest sources order[0 .. coop_n) one at a time from its own
    // queue head (coop_work) and runs each with the whole warp, its two heaps
    // in the block's shared memory; then, like every other warp, it runs one
    // source per lane from order[coop_n ..).
    int32_t coop_n;
    int32_t coop_warps;
    int32_t* coop_work;
    // 1: once the work queue is drained, a warp left with one running lane
    // finishes that lane's source in the cooperative form
    int32_t coop_tail;
};

template <class LaneType>
__device__ void record_stats(const LaneType& L, const PhaseOut& O, int v) {
    O.st_windows[v] = L.st_windows();
    O.st_maxq[v] = L.st_maxw();
    int f = 0;
    if (L.flags & kFlagQueueDrop) f |= 1;
    if (L.flags & kFlagRefOverflow) f |= 2;
    if (L.flags & kFlagWatchdog) f |= 4;
    if (L.flags & kFlagUndefined) f |= 8;
    O.st_flags[v] = f;
    atomicAdd(&O.acc[0], (unsigned long long)L.st_windows());
    atomicAdd(&O.acc[1], (unsigned long long)L.st_generated());
    atomicAdd(&O.acc[2], (unsigned long long)L.st_pseudos());
    atomicMax(reinterpret_cast<unsigned long long*>(&O.acc[3]), (unsigned long long)L.st_maxw());
    atomicMax(reinterpret_cast<unsigned long long*>(&O.acc[4]), (unsigned long long)L.st_maxp());
}

// End of the sources of the lanes in `amask` (they finished in this step):
// export each one's direct candidates.  BuildGeodesicPathTo
// (ICHDevice.cu:336-480) sets pathPassVert on its first hop already: through a
// vertex that is not the source (enterEdge starts at the vertex, or a window
// chain whose pseudo-source is another vertex), or through enterEdge -1.  A
// vertex at distance 0 has no key point at all.  The vertex list holds table
// slots and each vertex slot the split slot of its enter edge, so the walk is
// direct loads; the whole warp walks each finished lane's list 32 entries at a
// time (the other lanes would only wait), and a ballot keeps the candidates
// in list order.  Every lane of the warp calls it.
template <class LaneType>
__device__ void finish_warp(LaneType& L, const PhaseOut& O, int v, unsigned amask) {
    constexpr unsigned kFull = 0xFFFFFFFFu;
    const int lane = threadIdx.x & 31;
    const DevMesh& M = L.C.M;
    const int warp_base = blockIdx.x * blockDim.x + (threadIdx.x & ~31);
    unsigned todo = amask;
    while (todo) {
        const int o = __ffs(todo) - 1;
        todo &= todo - 1;
        // what only the owner knows: retry, pool space, statistics
        int skip = 0;
        unsigned long long base = 0;
        if (lane == o) {
            if (L.flags & kFlagCapacity) {
                const int k = atomicAdd(O.retry_n, 1);
                O.retry[k] = v;
                skip = 1;
            } else {
                base = atomicAdd(O.cand_used, (unsigned long long)L.vcount);
                record_stats(L, O, v);
                if (base + (unsigned long long)L.vcount > (unsigned long long)O.cand_cap) {
                    O.cand_n[v] = 0;  // the host sees cand_used > cand_cap and reruns with a larger pool
                    O.deg[v] = 0;
                    skip = 1;
                }
            }
        }
        if (__shfl_sync(kFull, skip, o)) continue;
        base = __shfl_sync(kFull, base, o);
        const int vo = __shfl_sync(kFull, v, o);
        const int vcount = __shfl_sync(kFull, L.vcount, o);
        const uint32_t ep = __shfl_sync(kFull, L.epoch, o);
        const size_t og = (size_t)(warp_base + o);
        const int32_t* VL = L.C.vlist + og * (size_t)L.C.vlimit;
        const VSlot* VT = L.C.vtab + (og << L.C.vcap_log2);
        const SSlot* ST = L.C.stab + (og << L.C.scap_log2);
        const uint32_t smask = (1u << L.C.scap_log2) - 1;
        int n = 0;
        bool undef = false;
        for (int i0 = 0; i0 < vcount; i0 += 32) {
            const int i = i0 + lane;
            bool direct = false;
            Cand c;
            if (i < vcount) {
                const VSlot e = VT[VL[i]];
                const int u = (int)e.key;
                const double d = e.dist;
                if (d != DBL_MAX && u != vo) {
                    c.u = u;
                    c.dist = d;
                    c.ee = -1;
                    c.x = 0.0;
                    if (d == 0.0) {
                        direct = true;
                    } else if (e.enter != -1) {
                        const int enter = e.enter;
                        const HeRec h = ld_he(M.he, enter);
                        if (h.v0 == u) {
                            direct = (h.v1 == vo);
                        } else {
                            int ss = e.sslot;
                            if (ss < 0) {  // the owner's split table, probed as Lane::sfind does
                                uint32_t hh = (((uint32_t)enter * 0x9E3779B1u) >> (32 - L.C.scap_log2));
                                for (;;) {
                                    const uint2 ke = *reinterpret_cast<const uint2*>(&ST[hh]);
                                    if (ke.y != ep) break;
                                    if (ke.x == (uint32_t)enter) {
                                        ss = (int)hh;
                                        break;
                                    }
                                    hh = (hh + 1) & smask;
                                }
                            }
                            const int psrc = ss < 0 ? -1 : ST[ss].psrc;
                            if ((unsigned)psrc >= (unsigned)M.nv) {
                                undef = true;
                            } else {
                                direct = (psrc == vo);
                                c.ee = enter;
                                c.x = ST[ss].x;
                            }
                        }
                    }
                }
            }
            const unsigned dm = __ballot_sync(kFull, direct);
            if (direct) O.cand[base + (unsigned long long)(n + __popc(dm & ((1u << lane) - 1u)))] = c;
            n += __popc(dm);
        }
        const bool anyu = __ballot_sync(kFull, undef) != 0;
        if (lane == o) {
            if (anyu) L.flags |= kFlagUndefined;
            O.cand_start[v] = (int64_t)base;
            O.cand_n[v] = n;
            O.deg[v] = min(n, L.C.K);
            if (L.flags & kFlagUndefined) O.st_flags[v] |= 8;
        }
    }
}

// Longest a lane waits for its action type to be chosen (iterations).

// Persistent batched build.  Each lane runs one source at a time and pulls
// the next from the device work queue.  Every iteration the warp votes: each
// lane's next action is a window pop, a pseudo-source pop or "source done"
// (export + start the next source); the action type held by the most lanes
// runs, the other lanes wait - at most C.max_wait iterations, after
// which the longest-waiting lane's type runs.  A lane's own sequence of
// actions is unchanged; only when it takes them is, so the rare, long paths
// (pseudo-source fans, exports) run with many lanes at once instead of one
// lane while 31 idle.
__global__ void SVG_ICH_BOUNDS k_ich_batched(LaneConfig C, PhaseOut O) {
    constexpr unsigned kFull = 0xFFFFFFFFu;
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    if (threadIdx.x < 32 && (int)blockIdx.x < O.coop_warps) {
        // Cooperative phase: the whole warp on one heavy source at a time,
        // its heaps in shared memory, its pool and tables in the scratch of
        // the warp's first lane.
        extern __shared__ __align__(16) unsigned char s_heaps[];
        const int wbase = gtid & ~31;
        CoopLane W(C, wbase);
        W.sheap = reinterpret_cast<WinEntry*>(s_heaps);
        for (;;) {
            int rc = 0;
            if ((threadIdx.x & 31) == 0) rc = atomicAdd(O.coop_work, 1);
            rc = __shfl_sync(kFull, rc, 0);
            if (rc >= O.coop_n) break;
            const int vc = O.order[rc];
            W.begin(vc, false);
            while (!W.step()) {
            }
            finish_warp(W, O, vc, 1u);  // every thread holds the source's state: lane 0 is its owner
        }
        if ((threadIdx.x & 31) == 0) W.save_epoch(wbase);
        __syncwarp();
    }
    Lane L(C, gtid);
    int r = O.coop_n + atomicAdd(O.work, 1);
    int v = r < O.nsrc ? O.order[r] : -1;
    if (v >= 0) L.begin(v, false);
    int waited = 0;
    int adopt = -1;
    for (;;) {
        const int act = v >= 0 ? L.template peek<SVG_ICH_INLINE_STALE>() : -1;
        const unsigned m0 = __ballot_sync(kFull, act == Lane::kActWindow);
        const unsigned m1 = __ballot_sync(kFull, act == Lane::kActPseudo);
        const unsigned m2 = __ballot_sync(kFull, act == Lane::kActDone);
        if ((m0 | m1 | m2) == 0) break;
        const unsigned starving = __ballot_sync(kFull, act >= 0 && waited >= C.max_wait);
        int chosen;
        if (starving) {
            chosen = __shfl_sync(kFull, act, __ffs(starving) - 1);
        } else {
            const int c0 = __popc(m0), c1 = __popc(m1), c2 = __popc(m2);
            chosen = (c0 >= c1 && c0 >= c2) ? Lane::kActWindow : (c1 >= c2 ? Lane::kActPseudo : Lane::kActDone);
        }
        if (O.coop_tail && m2 == 0 && __popc(m0 | m1) == 1 && __ballot_sync(kFull, v < 0) == ~(m0 | m1)) {
            // The queue is drained (every other lane found it empty) and one
            // lane still runs a source: the whole warp adopts it below.
            adopt = __ffs(m0 | m1) - 1;
            break;
        }
        const unsigned amask = chosen == Lane::kActWindow ? m0 : (chosen == Lane::kActPseudo ? m1 : m2);
        if (chosen == Lane::kActDone) finish_warp(L, O, v, amask);  // the whole warp exports
        if (act == chosen) {
            waited = 0;
            if (chosen == Lane::kActWindow) {
                L.act_window(amask);
            } else if (chosen == Lane::kActPseudo) {
                L.act_pseudo(amask);
            } else {
                r = O.coop_n + atomicAdd(O.work, 1);
                v = r < O.nsrc ? O.order[r] : -1;
                if (v >= 0) L.begin(v, false);
            }
        } else if (act >= 0) {
            ++waited;
        }
    }
    L.save_epoch(gtid);  // adoption below keeps lane `adopt`'s epoch: no begin() runs there
    if (adopt >= 0) {
        CoopLane W(C, blockIdx.x * blockDim.x + (threadIdx.x & ~31));
        W.adopt(L, adopt);
        while (!W.step()) {
        }
        finish_warp(W, O, __shfl_sync(kFull, v, adopt), 1u << adopt);  // lane `adopt`'s scratch; it owns it
    }
}

// BuildGeodesicPathTo(vertex) (ICHDevice.cu:336-480), the full back-trace the
// plain emission runs for every reached vertex.  Returns pathPassVert.
__device__ bool trace_full(Lane& L, int vert, uint32_t& se, double& sx, uint32_t& de, double& dx) {
    const DevMesh& M = L.C.M;
    bool pass = false;
    se = 0xFFFFFFFFu;
    de = 0xFFFFFFFFu;
    int curVert = vert;
    int guard = 0;
    for (;;) {
        int s = L.vfind(curVert);
        double d = s < 0 ? DBL_MAX : L.VT()[s].dist;
        if (d == 0.0) break;
        if (++guard > M.nf + 8) { L.flags |= kFlagWatchdog; return true; }
        int enterEdge = s < 0 ? -1 : L.VT()[s].enter;
        if (enterEdge == -1) {
            if (de == 0xFFFFFFFFu) { de = (uint32_t)__ldg(&M.vr[curVert].first); dx = 0.0; }
            else { se = (uint32_t)__ldg(&M.vr[curVert].first); sx = 0.0; }
            return true;
        }
        HeRec he = ld_he(M.he, enterEdge);
        if (he.v0 == curVert) {
            int nextVert = he.v1;
            if (nextVert != L.source) {
                if (de == 0xFFFFFFFFu) { de = (uint32_t)nxt(enterEdge); dx = 0.0; }
                else { se = (uint32_t)nxt(enterEdge); sx = 0.0; }
                pass = true;
            }
            curVert = nextVert;
            continue;
        }
        int ss = L.sfind(enterEdge);
        double gpos = ss < 0 ? DBL_MAX : L.ST()[ss].x;
        int psrc = ss < 0 ? -1 : L.ST()[ss].psrc;
        int gid = enterEdge;
        if (de == 0xFFFFFFFFu) { de = (uint32_t)gid; dx = gpos; }
        else { se = (uint32_t)gid; sx = gpos; }
        if ((unsigned)psrc >= (unsigned)M.nv || he.twin < 0) { L.flags |= kFlagUndefined; return true; }
        int opv = ld_he(M.he, nxt(he.twin)).v1;
        double2 last = ld_apex(M.geo, gid);
        double cx = he.len - gpos, cy = 0.0;
        HeRec hg = he;
        while (opv != psrc) {
            if (++guard > M.nf + 8) { L.flags |= kFlagWatchdog; return true; }
            int e0 = hg.twin, e1 = nxt(e0), e2 = nxt(e1);
            double L0 = ld_he(M.he, e0).len, L1 = ld_he(M.he, e1).len, L2 = ld_he(M.he, e2).len;
            double2 ov = ld_top(M.geo, e0);
            double s_ = gpos / L0, t_ = 1.0 - gpos / L0;
            double2 nl;
            if (to_left(ov.x, ov.y, last.x, last.y, cx, cy)) {
                double2 p0 = ld_apex(M.geo, e1);
                nl.x = p0.x * s_ + L1 * t_;
                nl.y = p0.y * s_ + 0.0 * t_;
                gpos = isect(last.x, last.y, cx, cy, L0, 0.0, ov.x, ov.y);
                gpos = (1.0 - gpos) * L1;
                gid = e1;
                cx = L1 - gpos;
            } else {
                double2 p1 = ld_apex(M.geo, e2);
                nl.x = 0.0 * s_ + p1.x * t_;
                nl.y = 0.0 * s_ + p1.y * t_;
                gpos = isect(last.x, last.y, cx, cy, ov.x, ov.y, 0.0, 0.0);
                gpos = (1.0 - gpos) * L2;
                gid = e2;
                cx = L2 - gpos;
            }
            cy = 0.0;
            last = nl;
            se = (uint32_t)gid;
            sx = gpos;
            hg = ld_he(M.he, gid);
            if (hg.twin < 0) { L.flags |= kFlagUndefined; return true; }
            opv = ld_he(M.he, nxt(hg.twin)).v1;
        }
        if (opv != L.source) {
            se = (uint32_t)__ldg(&M.vr[opv].first);
            sx = 0.0;
            pass = true;
        }
        curVert = opv;
    }
    return pass;
}

struct PlainOut {
    const int32_t* order;
    int32_t nsrc;
    int32_t* tails;        // per row
    int32_t* adj;          // nsrc*K padded rows
    double* dist;
    PathEnd* path;
    PhaseOut stats;
};

// constructSVG (SVG.cu:9-96): one source per thread, grid-stride.
__global__ void __launch_bounds__(128) k_ich_plain(LaneConfig C, PlainOut O) {
    int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    int stride = gridDim.x * blockDim.x;
    Lane L(C, gtid);
    const int K = C.K;
    for (int r = gtid; r < O.nsrc; r += stride) {
        int v = O.order[r];
        L.begin(v, true);
        while (!L.step()) {
        }
        int tail = 0;
        size_t row = (size_t)r * K;
        if (!(L.flags & kFlagCapacity)) {
            for (int j = 0; j < C.M.nv && K > 0; ++j) {
                double d = L.vdist(j);
                if (d == DBL_MAX || j == v) continue;
                uint32_t se, de;
                double sx = 0.0, dx = 0.0;
                if (trace_full(L, j, se, sx, de, dx)) continue;
                if (se == 0xFFFFFFFFu) { se = de; sx = dx; }
                O.adj[row + tail] = j;
                O.dist[row + tail] = d;
                if (O.path) {
                    PathEnd pe;
                    pe.src_edge = se; pe.dst_edge = de; pe.src_x = sx; pe.dst_x = dx;
                    O.path[row + tail] = pe;
                }
                if (++tail == K) break;
            }
        }
        O.tails[r] = tail;
        O.stats.deg[v] = tail;
        if (L.flags & kFlagCapacity) {
            int k = atomicAdd(O.stats.retry_n, 1);
            O.stats.retry[k] = v;
        } else {
            record_stats(L, O.stats, v);
        }
    }
}

struct EmitParams {
    DevMesh M;
    int32_t K;
    int32_t nv;
    const int32_t* order;
    int32_t nsrc;
    const Cand* cand;
    const int64_t* cand_start;
    const int32_t* cand_n;
    const int64_t* off;
    int32_t* adj;
    double* dist;
    PathEnd* path;
    int32_t* st_flags;
    int32_t smax;            // sort capacity per warp (power of two)
};

// Path ends of the emitted rows (k_emit with SVG_SPLIT_TRACE): one thread per
// SVG edge whose path has a key point walks back from it to the source
// (BuildGeodesicPathTo, ICHDevice.cu:336-480).  A walk is a chain of dependent
// loads; run apart from the sort, with small blocks and few registers, many
// more of them are in flight than inside k_emit's warps.
__global__ void __launch_bounds__(256, SVG_TRACE_MIN_BLOCKS) k_trace(DevMesh M, PathEnd* path, int64_t nnz, int32_t* st_flags) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += stride) {
        PathEnd pe = path[e];
        if (!(pe.src_x < 0.0)) continue;
        const int v = (int)pe.src_edge;
        int fl = 0;
        trace_direct(M, v, (int)pe.dst_edge, pe.dst_x, pe.src_edge, pe.src_x, fl);
        if (pe.src_edge == 0xFFFFFFFFu) {
            pe.src_edge = pe.dst_edge;
            pe.src_x = pe.dst_x;
        }
        path[e] = pe;
        if (fl) atomicOr(&st_flags[v], (fl & kFlagWatchdog) ? 4 : 8);
    }
}

// Warp-per-source emission.
__global__ void __launch_bounds__(256) k_emit(EmitParams P) {
    extern __shared__ unsigned long long sm_keys[];
    int lane = threadIdx.x & 31;
    int wib = threadIdx.x >> 5;
    unsigned long long* keys = sm_keys + (size_t)wib * P.smax;
    int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int nw = (gridDim.x * blockDim.x) >> 5;
    for (int r = gw; r < P.nsrc; r += nw) {
        int v = P.order[r];
        int n = P.cand_n[v];
        if (n <= 0) continue;
        int64_t start = P.cand_start[v];
        int N = 32;
        while (N < n) N <<= 1;
        if (N > P.smax) {  // cannot happen: smax covers the largest vertex list
            if (lane == 0) P.st_flags[v] |= 8;
            continue;
        }
        for (int i = lane; i < N; i += 32)
            keys[i] = i < n ? ((unsigned long long)(uint32_t)P.cand[start + i].u << 32) | (uint32_t)i
                            : ~0ull;
        __syncwarp();
        for (int k = 2; k <= N; k <<= 1) {
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int i = lane; i < N; i += 32) {
                    int ixj = i ^ j;
                    if (ixj > i) {
                        unsigned long long a = keys[i], b = keys[ixj];
                        bool up = (i & k) == 0;
                        if ((a > b) == up) {
                            keys[i] = b;
                            keys[ixj] = a;
                        }
                    }
                }
                __syncwarp();
            }
        }
        int deg = min(n, P.K);
        int64_t base = P.off[v];
        int fl = 0;
        for (int i = lane; i < deg; i += 32) {
            int idx = (int)(keys[i] & 0xFFFFFFFFu);
            Cand c = P.cand[start + idx];
            P.adj[base + i] = c.u;
            P.dist[base + i] = c.dist;
            if (P.path) {
                PathEnd pe;
                if (c.ee < 0) {
                    pe.src_edge = pe.dst_edge = 0xFFFFFFFFu;
                    pe.src_x = pe.dst_x = 0.0;
                } else {
                    pe.dst_edge = (uint32_t)c.ee;
                    pe.dst_x = c.x;
#if SVG_SPLIT_TRACE
                    // the path's first key point is traced by k_trace: the
                    // source in src_edge, a negative src_x marks it pending
                    pe.src_edge = (uint32_t)v;
                    pe.src_x = -1.0;
#else
                    trace_direct(P.M, v, c.ee, c.x, pe.src_edge, pe.src_x, fl);
                    if (pe.src_edge == 0xFFFFFFFFu) {
                        pe.src_edge = pe.dst_edge;
                        pe.src_x = pe.dst_x;
                    }
#endif
                }
                P.path[base + i] = pe;
            }
        }
        if (fl) atomicOr(&P.st_flags[v], (fl & kFlagWatchdog) ? 4 : 8);
        __syncwarp();
    }
}

// Pack padded rows (plain build) into CSR.
__global__ void k_compact(const int32_t* order, int32_t nsrc, int32_t K, const int32_t* tails,
                          const int32_t* padj, const double* pdist, const PathEnd* ppath, const int64_t* off,
                          int32_t* adj, double* dist, PathEnd* path) {
    int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    int nw = (gridDim.x * blockDim.x) >> 5;
    for (int r = gw; r < nsrc; r += nw) {
        int v = order[r];
        int t = tails[r];
        int64_t b = off[v];
        size_t row = (size_t)r * K;
        for (int i = lane; i < t; i += 32) {
            adj[b + i] = padj[row + i];
            dist[b + i] = pdist[row + i];
            if (path) path[b + i] = ppath[row + i];
        }
    }
}

__global__ void k_iota(int32_t* o, int32_t n, int32_t base) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) o[i] = base + i;
}

// ------------------------------------------------------------------ host

namespace {

struct Layout {
    int32_t lanes = 0, wphys = 0, pphys = 0, vcap_log2 = 0, scap_log2 = 0, vlimit = 0;
    bool operator==(const Layout& o) const {
        return lanes == o.lanes && wphys == o.wphys && pphys == o.pphys && vcap_log2 == o.vcap_log2 &&
               scap_log2 == o.scap_log2 && vlimit == o.vlimit;
    }
};

size_t align_up(size_t x, size_t a = 256) { return (x + a - 1) / a * a; }

// heap entries per lane: the three-level sift-down reads up to index cap + 7
// (the stride leaves 16 entries past the capacity)
int heap_stride(int cap) { return (cap + 16 + 3) / 4 * 4; }

// k_trace's grid: one thread per edge, at most 4,096 blocks of 256 (grid-stride)
int trace_blocks(int64_t nnz) { return (int)std::max<int64_t>(1, std::min<int64_t>((nnz + 255) / 256, 4096)); }

size_t lane_bytes(const Layout& l) {
    size_t b = 0;
    b += (size_t)heap_stride(l.wphys) * sizeof(WinEntry);
    b += (size_t)l.wphys * sizeof(WinPay);
    b += (size_t)l.wphys * sizeof(uint16_t);
    b += (size_t)heap_stride(l.pphys) * sizeof(PsEntry);
    b += ((size_t)1 << l.vcap_log2) * sizeof(VSlot);
    b += (size_t)l.vlimit * sizeof(int32_t);
    b += ((size_t)1 << l.scap_log2) * sizeof(SSlot);
    b += sizeof(uint32_t);
    return b;
}

// Lane scratch, kept across builds; zeroed when its layout changes so epoch
// stamps never alias.
struct Arena {
    DevBuf buf;
    Layout layout;
};
Arena g_arena[2];  // [0] main pass, [1] retry pass with larger tables

void carve(Arena& A, const Layout& l, LaneConfig& C, cudaStream_t st) {
    size_t lanes = (size_t)l.lanes;
    size_t sz[7] = {
        align_up(lanes * heap_stride(l.wphys) * sizeof(WinEntry)),
        align_up(lanes * l.wphys * sizeof(WinPay)),
        align_up(lanes * l.wphys * sizeof(uint16_t)),
        align_up(lanes * heap_stride(l.pphys) * sizeof(PsEntry)),
        align_up(lanes * ((size_t)1 << l.vcap_log2) * sizeof(VSlot)),
        align_up(lanes * l.vlimit * sizeof(int32_t)),
        align_up(lanes * ((size_t)1 << l.scap_log2) * sizeof(SSlot)),
    };
    size_t ep = align_up(lanes * sizeof(uint32_t));
    size_t total = ep;
    for (size_t s : sz) total += s;
    bool fresh = !(A.layout == l) || A.buf.bytes < total;
    if (A.buf.bytes < total) A.buf.reserve(total);
    char* p = A.buf.as<char>();
    C.wheap = reinterpret_cast<WinEntry*>(p); p += sz[0];
    C.wpool = reinterpret_cast<WinPay*>(p); p += sz[1];
    C.wfree = reinterpret_cast<uint16_t*>(p); p += sz[2];
    C.pheap = reinterpret_cast<PsEntry*>(p); p += sz[3];
    C.vtab = reinterpret_cast<VSlot*>(p); p += sz[4];
    C.vlist = reinterpret_cast<int32_t*>(p); p += sz[5];
    C.stab = reinterpret_cast<SSlot*>(p); p += sz[6];
    C.epochs = reinterpret_cast<uint32_t*>(p);
    if (fresh) {
        SVG_CUDA(cudaMemsetAsync(C.vtab, 0, sz[4], st));
        SVG_CUDA(cudaMemsetAsync(C.stab, 0, sz[6], st));
        SVG_CUDA(cudaMemsetAsync(C.epochs, 0, ep, st));
        A.layout = l;
    }
}

int ilog2_ceil(int64_t x) {
    int k = 0;
    while (((int64_t)1 << k) < x) ++k;
    return k;
}

}  // namespace

// ------------------------------------------------------- build as a graph
//
// A batched build whose sources all fit the first pass (no retry) and whose
// candidate pool was large enough can be replayed: the device work is one
// sequence of memsets, k_ich_batched, the offsets scan, k_emit and the copies
// of the CSR and per-source counters into the graph's own buffers, over
// buffers whose sizes the first build fixed.  It is captured once, kept with
// the mesh, and launched as one graph by later builds with the same options;
// only the copies' destinations change from launch to launch.  A replay reads
// back a status block (retry count, candidate pool use, edge count, counters)
// and falls back to the ordinary build if the sizes no longer hold.
struct BuildGraph {
    svg_build_opts opts{};
    Layout lay;
    void* arena = nullptr;
    int32_t nv = 0, nsrc = 0, sb = 0, se = 0;
    int64_t nnz = 0, cand_cap = 0;
    int32_t coop_n = 0, coop_warps = 0;
    int64_t scratch_bytes = 0;
    bool with_paths = false;
    DevBuf order, misc, cand, candstart, stats, off, adj, dist, paths, tmp;
    int32_t* d_retry_n = nullptr;
    unsigned long long* d_acc = nullptr;  // acc[0..7], cand_used at acc[8]
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaGraphNode_t cp_off{}, cp_adj{}, cp_dist{}, cp_paths{}, cp_stats{};
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    ~BuildGraph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
    }
};

namespace {
// Options that decide a build's device work (all but the graph switch itself).
bool same_build_options(const svg_build_opts& a, const svg_build_opts& b) {
    return a.K == b.K && a.split_coef == b.split_coef && a.vert_coef == b.vert_coef &&
           a.win_queue_cap == b.win_queue_cap && a.pseudo_queue_cap == b.pseudo_queue_cap && a.mode == b.mode &&
           a.threads_per_block == b.threads_per_block && a.blocks == b.blocks && a.with_paths == b.with_paths &&
           a.heavy_first == b.heavy_first && a.hbm_budget == b.hbm_budget && a.source_begin == b.source_begin &&
           a.source_end == b.source_end && a.coop_sources == b.coop_sources && a.coop_warps == b.coop_warps &&
           a.vote_wait == b.vote_wait && a.heavy_waves == b.heavy_waves && a.heap_factor == b.heap_factor &&
           a.coop_tail == b.coop_tail;
}
}  // namespace

namespace {
// Options a build runs with: the caller's, or, with autotune set, the
// launch parameters svg_build_autotune cached on the mesh for this K.
svg_build_opts effective_options(const svg_mesh* m, const svg_build_opts& o) {
    svg_build_opts e = o;
    if (o.autotune && o.mode != SVG_BUILD_PLAIN) {
        for (const auto& t : m->tuned)
            if (t.K == o.K) {
                e.coop_sources = t.opts.coop_sources;
                e.coop_warps = t.opts.coop_warps;
                e.vote_wait = t.opts.vote_wait;
                e.heavy_waves = t.opts.heavy_waves;
                e.heap_factor = t.opts.heap_factor;
                e.blocks = t.opts.blocks;
                e.coop_tail = t.opts.coop_tail;
            }
    }
    if (e.vote_wait <= 0) e.vote_wait = 8;
    if (e.heavy_waves <= 0) e.heavy_waves = 2;
    if (e.heap_factor <= 0) e.heap_factor = 3;
    return e;
}
}  // namespace

namespace {
// Flag tallies of a finished build; per-source costs kept on the mesh for
// the next build's order.
void record_counts(svg_mesh* m, svg_graph* g, int32_t K, int32_t sb, int32_t se, bool plain) {
    const int32_t nv = g->nv;
    svg_build_stats& S = g->stats;
    std::vector<int32_t> fl((size_t)nv);
    SVG_CUDA(cudaMemcpy(fl.data(), g->st_flags, sizeof(int32_t) * (size_t)nv, cudaMemcpyDeviceToHost));
    if (!plain) {
        std::vector<int32_t> w((size_t)nv);
        SVG_CUDA(cudaMemcpy(w.data(), g->st_windows, sizeof(int32_t) * (size_t)nv, cudaMemcpyDeviceToHost));
        if (m->cost_K != K || (int32_t)m->cost.size() != nv) {
            m->cost.assign((size_t)nv, 0);
            m->cost_K = K;
            m->cost_probe = false;
        }
        for (int32_t v = sb; v < se; ++v) m->cost[(size_t)v] = w[(size_t)v];
        if (sb == 0 && se == nv) m->cost_probe = false;
    }
    for (int32_t f : fl) {
        if (f & 1) ++S.queue_drop_sources;
        if (f & 2) ++S.ref_overflow_sources;
        if (f & 4) ++S.watchdog_sources;
        if (f & 8) ++S.undefined_sources;
    }
}

// A replay of the mesh's captured build: false (nothing of g kept) when
// there is none for these options, the lane scratch has moved, or the
// sources no longer fit the captured sizes.
bool replay_graph(svg_mesh* m, const svg_build_opts& o, svg_graph* g) {
    BuildGraph* bg = m->build_graph.get();
    if (!bg || !same_build_options(bg->opts, o)) return false;
    if (!(g_arena[0].layout == bg->lay) || g_arena[0].buf.p != bg->arena) return false;
    cudaStream_t st = lib_stream();
    const int32_t nv = bg->nv;
    const size_t E = (size_t)std::max<int64_t>(bg->nnz, 1);
    g->nv = nv;
    g->K = o.K;
    g->with_paths = bg->with_paths;
    g->st_windows = dev_alloc_n<int32_t>((size_t)nv * 3);
    g->st_maxq = g->st_windows + nv;
    g->st_flags = g->st_maxq + nv;
    g->off = dev_alloc_n<int64_t>((size_t)nv + 1);
    g->adj = dev_alloc_n<int32_t>(E);
    g->dist = dev_alloc_n<double>(E);
    if (g->with_paths) g->paths = dev_alloc(sizeof(PathEnd) * E);
    const auto D2D = cudaMemcpyDeviceToDevice;
    SVG_CUDA(cudaGraphExecMemcpyNodeSetParams1D(bg->exec, bg->cp_off, g->off, bg->off.p, sizeof(int64_t) * ((size_t)nv + 1), D2D));
    SVG_CUDA(cudaGraphExecMemcpyNodeSetParams1D(bg->exec, bg->cp_adj, g->adj, bg->adj.p, sizeof(int32_t) * E, D2D));
    SVG_CUDA(cudaGraphExecMemcpyNodeSetParams1D(bg->exec, bg->cp_dist, g->dist, bg->dist.p, sizeof(double) * E, D2D));
    if (g->with_paths)
        SVG_CUDA(cudaGraphExecMemcpyNodeSetParams1D(bg->exec, bg->cp_paths, g->paths, bg->paths.p, sizeof(PathEnd) * E, D2D));
    SVG_CUDA(cudaGraphExecMemcpyNodeSetParams1D(bg->exec, bg->cp_stats, g->st_windows, bg->stats.p,
                                                 sizeof(int32_t) * 3 * (size_t)nv, D2D));
    cudaEvent_t e0, e1;
    SVG_CUDA(cudaEventCreate(&e0));
    SVG_CUDA(cudaEventCreate(&e1));
    SVG_CUDA(cudaEventRecord(e0, st));
    SVG_CUDA(cudaGraphLaunch(bg->exec, st));
    SVG_CUDA(cudaEventRecord(e1, st));
    int32_t retry_n = 0;
    unsigned long long acc[9] = {0};
    int64_t nnz = 0;
    SVG_CUDA(cudaMemcpyAsync(&retry_n, bg->d_retry_n, sizeof(retry_n), cudaMemcpyDeviceToHost, st));
    SVG_CUDA(cudaMemcpyAsync(acc, bg->d_acc, sizeof(acc), cudaMemcpyDeviceToHost, st));
    SVG_CUDA(cudaMemcpyAsync(&nnz, bg->off.as<int64_t>() + nv, sizeof(nnz), cudaMemcpyDeviceToHost, st));
    SVG_CUDA(cudaStreamSynchronize(st));
    float ms = 0.f, ms_ich = 0.f, ms_emit = 0.f;
    SVG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    SVG_CUDA(cudaEventElapsedTime(&ms_ich, bg->ev[0], bg->ev[1]));
    SVG_CUDA(cudaEventElapsedTime(&ms_emit, bg->ev[2], bg->ev[3]));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (retry_n != 0 || (int64_t)acc[8] > bg->cand_cap || nnz != bg->nnz) {
        free_graph_device(g);
        return false;
    }
    g->nnz = nnz;
    svg_build_stats& S = g->stats;
    S = svg_build_stats{};
    S.ms_ich = ms_ich;
    S.ms_emit = ms_emit;
    S.ms_total = ms;
    S.windows = (int64_t)acc[0];
    S.windows_generated = (int64_t)acc[1];
    S.pseudo_sources = (int64_t)acc[2];
    S.max_win_queue = (int32_t)acc[3];
    S.max_pseudo_queue = (int32_t)acc[4];
    S.edges = nnz;
    S.sources = bg->nsrc;
    S.launches = (SVG_SPLIT_TRACE && bg->opts.with_paths) ? 4 : 3;  // k_ich_batched, the offsets scan,
                                                                     // k_emit (and k_trace), in one graph launch
    S.scratch_bytes = bg->scratch_bytes;
    S.coop_sources = bg->coop_n;
    S.coop_warps = bg->coop_warps;
    S.graph_replayed = 1;
    record_counts(m, g, o.K, bg->sb, bg->se, false);
    return true;
}

struct CapturePlan {
    LaneConfig C;
    PhaseOut O;
    int blocks = 0, tpb = 0;
    size_t coop_smem = 0;
    const int32_t* d_order = nullptr;
    int32_t nsrc = 0, nv = 0, sb = 0, se = 0;
    int64_t cap = 0, nnz = 0;
    size_t tmp_bytes = 0, misc_bytes = 0, retry_bytes = 0;
    int eb = 0, wpb = 0, smax = 32;
    size_t emit_smem = 0;
    bool with_paths = false;
    Layout lay;
    int64_t scratch_bytes = 0;
    int32_t coop_n = 0, coop_warps = 0;
};

// Capture the device work of the build just finished (plan P, result g) as a
// graph over buffers of its own, kept with the mesh.  g's buffers stand in as
// the copies' destinations until a replay retargets them.
void capture_graph(svg_mesh* m, const svg_build_opts& o, const CapturePlan& P, svg_graph* g) {
    auto bg = std::make_shared<BuildGraph>();
    cudaStream_t st = lib_stream();
    const int32_t nv = P.nv;
    const size_t E = (size_t)std::max<int64_t>(P.nnz, 1);
    bg->opts = o;
    bg->lay = P.lay;
    bg->arena = g_arena[0].buf.p;
    bg->nv = nv;
    bg->nsrc = P.nsrc;
    bg->sb = P.sb;
    bg->se = P.se;
    bg->nnz = P.nnz;
    bg->cand_cap = P.cap;
    bg->coop_n = P.coop_n;
    bg->coop_warps = P.coop_warps;
    bg->scratch_bytes = P.scratch_bytes;
    bg->with_paths = P.with_paths;
    bg->order.reserve(sizeof(int32_t) * (size_t)P.nsrc);
    bg->misc.reserve(P.misc_bytes);
    bg->cand.reserve(sizeof(Cand) * (size_t)P.cap);
    bg->candstart.reserve(sizeof(int64_t) * ((size_t)nv + 1));
    bg->stats.reserve(sizeof(int32_t) * 3 * (size_t)nv);
    bg->off.reserve(sizeof(int64_t) * ((size_t)nv + 1));
    bg->adj.reserve(sizeof(int32_t) * E);
    bg->dist.reserve(sizeof(double) * E);
    if (P.with_paths) bg->paths.reserve(sizeof(PathEnd) * E);
    bg->tmp.reserve(P.tmp_bytes + 16);
    SVG_CUDA(cudaMemcpyAsync(bg->order.p, P.d_order, sizeof(int32_t) * (size_t)P.nsrc, cudaMemcpyDeviceToDevice, st));
    SVG_CUDA(cudaStreamSynchronize(st));
    // the misc block laid out as the ordinary build lays it out
    char* mp = bg->misc.as<char>();
    int32_t* d_work = reinterpret_cast<int32_t*>(mp);
    bg->d_retry_n = d_work + 1;
    bg->d_acc = reinterpret_cast<unsigned long long*>(mp + 64);
    int32_t* d_cand_n = reinterpret_cast<int32_t*>(mp + 256 + P.retry_bytes);
    int32_t* d_deg = d_cand_n + align_up(sizeof(int32_t) * ((size_t)nv + 1)) / sizeof(int32_t);
    int32_t* st_base = bg->stats.as<int32_t>();
    PhaseOut O = P.O;
    O.order = bg->order.as<int32_t>();
    O.work = d_work;
    O.retry_n = bg->d_retry_n;
    O.retry = reinterpret_cast<int32_t*>(mp + 256);
    O.cand = bg->cand.as<Cand>();
    O.cand_cap = P.cap;
    O.cand_start = bg->candstart.as<int64_t>();
    O.cand_used = bg->d_acc + 8;
    O.cand_n = d_cand_n;
    O.deg = d_deg;
    O.st_windows = st_base;
    O.st_maxq = st_base + nv;
    O.st_flags = st_base + 2 * (size_t)nv;
    O.acc = bg->d_acc;
    O.coop_work = d_work + 4;
    EmitParams Em{};
    Em.M = P.C.M;
    Em.K = P.C.K;
    Em.nv = nv;
    Em.order = O.order;
    Em.nsrc = P.nsrc;
    Em.cand = O.cand;
    Em.cand_start = O.cand_start;
    Em.cand_n = d_cand_n;
    Em.off = bg->off.as<int64_t>();
    Em.adj = bg->adj.as<int32_t>();
    Em.dist = bg->dist.as<double>();
    Em.path = P.with_paths ? bg->paths.as<PathEnd>() : nullptr;
    Em.st_flags = O.st_flags;
    Em.smax = P.smax;
    for (auto& e : bg->ev) SVG_CUDA(cudaEventCreate(&e));
    cudaStream_t cs;
    SVG_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaGraph_t graph = nullptr;
    try {
        SVG_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
        SVG_CUDA(cudaEventRecordWithFlags(bg->ev[0], cs, cudaEventRecordExternal));
        SVG_CUDA(cudaMemsetAsync(bg->misc.p, 0, P.misc_bytes, cs));
        SVG_CUDA(cudaMemsetAsync(bg->stats.p, 0, sizeof(int32_t) * 3 * (size_t)nv, cs));
        k_ich_batched<<<P.blocks, P.tpb, P.coop_smem, cs>>>(P.C, O);
        SVG_CUDA(cudaEventRecordWithFlags(bg->ev[1], cs, cudaEventRecordExternal));
        size_t tb = P.tmp_bytes;
        SVG_CUDA(cub::DeviceScan::ExclusiveSum(bg->tmp.p, tb, d_deg, bg->off.as<int64_t>(), nv + 1, cs));
        SVG_CUDA(cudaEventRecordWithFlags(bg->ev[2], cs, cudaEventRecordExternal));
        k_emit<<<P.eb, P.wpb * 32, P.emit_smem, cs>>>(Em);
        if (SVG_SPLIT_TRACE && P.with_paths && P.nnz > 0)
            k_trace<<<trace_blocks(P.nnz), 256, 0, cs>>>(P.C.M, Em.path, P.nnz, Em.st_flags);
        SVG_CUDA(cudaEventRecordWithFlags(bg->ev[3], cs, cudaEventRecordExternal));
        SVG_CUDA(cudaStreamEndCapture(cs, &graph));
    } catch (...) {
        cudaStreamEndCapture(cs, &graph);
        if (graph) cudaGraphDestroy(graph);
        cudaStreamDestroy(cs);
        cudaGetLastError();
        throw;
    }
    cudaStreamDestroy(cs);
    bg->graph = graph;
    // the captured sequence is one chain: its last node precedes the copies
    size_t n = 0;
    SVG_CUDA(cudaGraphGetNodes(graph, nullptr, &n));
    std::vector<cudaGraphNode_t> nodes(n);
    SVG_CUDA(cudaGraphGetNodes(graph, nodes.data(), &n));
    cudaGraphNode_t leaf = nullptr;
    for (auto nd : nodes) {
        size_t d = 0;
        SVG_CUDA(cudaGraphNodeGetDependentNodes(nd, nullptr, &d));
        if (d == 0) leaf = nd;
    }
    if (!leaf) throw SvgError{SVG_ERR_STATE, "graph capture: no last node"};
    const auto D2D = cudaMemcpyDeviceToDevice;
    SVG_CUDA(cudaGraphAddMemcpyNode1D(&bg->cp_off, graph, &leaf, 1, g->off, bg->off.p, sizeof(int64_t) * ((size_t)nv + 1), D2D));
    SVG_CUDA(cudaGraphAddMemcpyNode1D(&bg->cp_adj, graph, &leaf, 1, g->adj, bg->adj.p, sizeof(int32_t) * E, D2D));
    SVG_CUDA(cudaGraphAddMemcpyNode1D(&bg->cp_dist, graph, &leaf, 1, g->dist, bg->dist.p, sizeof(double) * E, D2D));
    if (P.with_paths)
        SVG_CUDA(cudaGraphAddMemcpyNode1D(&bg->cp_paths, graph, &leaf, 1, g->paths, bg->paths.p, sizeof(PathEnd) * E, D2D));
    SVG_CUDA(cudaGraphAddMemcpyNode1D(&bg->cp_stats, graph, &leaf, 1, g->st_windows, bg->stats.p,
                                      sizeof(int32_t) * 3 * (size_t)nv, D2D));
    SVG_CUDA(cudaGraphInstantiate(&bg->exec, graph, 0));
    m->build_graph = bg;
}
}  // namespace

svg_status run_build(svg_mesh* m, const svg_build_opts& o_in, svg_graph* g) {
    const svg_build_opts o = effective_options(m, o_in);
    upload_mesh(m);
    if (o.graph && o.mode != SVG_BUILD_PLAIN && replay_graph(m, o, g)) return SVG_OK;
    cudaStream_t st = lib_stream();
    const HostMesh& H = m->h;
    const int32_t nv = H.nv;
    const int32_t K = o.K;
    int32_t sb = o.source_begin, se = o.source_end;
    if (sb == 0 && se == 0) se = nv;
    if (sb < 0 || se > nv || sb > se) throw SvgError{SVG_ERR_ARG, "source range outside [0, nv]"};
    if (K <= 0 && K != -1) throw SvgError{SVG_ERR_ARG, "K must be positive"};
    if (K == -1) throw SvgError{SVG_ERR_ARG, "exhaustive ICH (K=-1) is not a build mode"};
    if (o.win_queue_cap < 1 || o.win_queue_cap > 65535 || o.pseudo_queue_cap < 1)
        throw SvgError{SVG_ERR_ARG, "queue capacities must be in [1, 65535]"};
    const int32_t nsrc = se - sb;
    const bool plain = o.mode == SVG_BUILD_PLAIN;
    // heavy_first 2 on a mesh with no cost record at this K: a probe build at
    // K/10 (a few per cent of the work) supplies the per-source estimate.  It
    // runs before this build takes the scratch arena, which the probe reuses.
    // The order only pays where a lane gets few sources, so that the last,
    // heaviest ones set the build's length: up to kProbeSourcesPerLane per
    // lane of a full launch (measured: 6 % faster on a 72.9K-vertex height
    // field at K = 500 with 1.9 sources per lane, 4 % slower on a 750K-vertex
    // torus with 20).
    constexpr int kProbeSourcesPerLane = 4;
    int probe_lanes = 0;
    if (!plain && o.heavy_first == 2) {
        int per_sm = 0, dev0 = 0, sms = 0;
        SVG_CUDA(cudaGetDevice(&dev0));
        SVG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev0));
        SVG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_ich_batched, 128, 0));
        probe_lanes = std::max(1, per_sm) * sms * 128;
    }
    if (!plain && o.heavy_first == 2 && nsrc > 0 && K >= 160 &&
        (int64_t)nsrc <= (int64_t)kProbeSourcesPerLane * probe_lanes &&
        !(m->cost_K == K && (int32_t)m->cost.size() == nv)) {
        svg_build_opts po = o;
        po.K = K / 10;
        po.heavy_first = 0;
        po.with_paths = 0;
        svg_graph pg;
        pg.mesh = m;
        try {
            run_build(m, po, &pg);
        } catch (...) {
            free_graph_device(&pg);
            throw;
        }
        free_graph_device(&pg);
        if ((int32_t)m->cost.size() == nv) {
            m->cost_K = K;  // the probe's costs stand in for K's
            m->cost_probe = true;
        }
    }

    int dev = 0;
    SVG_CUDA(cudaGetDevice(&dev));
    static thread_local int prop_dev = -1;
    static thread_local cudaDeviceProp prop;
    if (prop_dev != dev) {
        SVG_CUDA(cudaGetDeviceProperties(&prop, dev));
        prop_dev = dev;
    }

    LaneConfig C{};
    C.M = m->d.view();
    C.K = K;
    C.wcap = o.win_queue_cap;
    C.pcap = o.pseudo_queue_cap;
    // Physical heaps of the first pass sized by K (observed high-water marks:
    // windows up to ~2.3K, pseudo-sources up to ~1.3K); a source that needs more is re-run
    // by the retry pass with physical = logical capacity.  The plain build
    // always uses the full capacity.
    C.wphys = plain ? C.wcap
                    : std::min<int32_t>(C.wcap,
                                        std::max<int32_t>(128, (int32_t)(((int64_t)o.heap_factor * K + 63) / 64 * 64)));
    C.pphys = plain ? C.pcap : std::min<int32_t>(C.pcap, std::max<int32_t>(128, (K + K / 2 + 64 + 63) / 64 * 64));
    C.wstride = heap_stride(C.wphys);
    C.pstride = heap_stride(C.pphys);
    C.vref = (uint32_t)K * o.vert_coef;
    C.sref = (uint32_t)K * o.split_coef;
    C.watchdog = (int64_t)1 << 26;
    C.max_wait = o.vote_wait;
    Layout lay;
    lay.wphys = C.wphys;
    lay.pphys = C.pphys;
    lay.vcap_log2 = std::max(6, ilog2_ceil(2 * ((int64_t)C.vref + 1))) + SVG_TABLE_SHIFT;
    lay.scap_log2 = std::max(8, ilog2_ceil(8 * (int64_t)K)) + SVG_SPLIT_SHIFT;  // split entries reach ~1.6x the vertices
    lay.vlimit = (int32_t)(((int64_t)3 << lay.vcap_log2) / 4);
    C.vcap_log2 = lay.vcap_log2;
    C.scap_log2 = lay.scap_log2;
    C.vlimit = lay.vlimit;
    C.slimit = (int32_t)(((int64_t)3 << lay.scap_log2) / 4);

    size_t freeb = 0, totalb = 0;
    SVG_CUDA(cudaMemGetInfo(&freeb, &totalb));
    int64_t budget = o.hbm_budget > 0 ? o.hbm_budget : (int64_t)((double)freeb * 0.5);

    int tpb = o.threads_per_block > 0 ? o.threads_per_block : 128;
    if (tpb % 32 != 0 || tpb > 128) throw SvgError{SVG_ERR_ARG, "threads_per_block must be a multiple of 32, <= 128"};
    int blocks = o.blocks;
    if (plain) {
        if (blocks <= 0) blocks = 64;  // SVG_BLOCK_NUM (SVG.cuh:10)
        if (o.threads_per_block <= 0) tpb = 128;  // SVG_THREAD_NUM
    } else if (blocks <= 0) {
        int per_sm = 0;
        SVG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_ich_batched, tpb, 0));
        blocks = std::max(1, per_sm) * prop.multiProcessorCount;
    }
    int64_t want_blocks = (nsrc + tpb - 1) / tpb;
    if (!plain) blocks = (int)std::min<int64_t>(blocks, std::max<int64_t>(1, want_blocks));
    lay.lanes = blocks * tpb;
    while (lay.lanes > 32 && (int64_t)(lane_bytes(lay) * lay.lanes) > budget) {
        blocks = std::max(1, blocks / 2);
        lay.lanes = blocks * tpb;
    }
    if ((int64_t)(lane_bytes(lay) * lay.lanes) > budget)
        throw SvgError{SVG_ERR_NOMEM, "HBM budget too small for one block of build lanes"};

    carve(g_arena[0], lay, C, st);

    // per-build buffers
    DevBuf b_order, b_misc, b_cand, b_candstart;
    int32_t coop_n = 0, coop_warps = 0;
    // what a capture of this build as a graph needs (see BuildGraph)
    size_t cap_coop_smem = 0, cap_emit_smem = 0;
    int cap_eb = 0, cap_wpb = 0, cap_attempts = 0;
    int64_t cap_pool = 0;
    b_order.reserve(sizeof(int32_t) * (size_t)std::max(nsrc, 1));
    int32_t* d_order = b_order.as<int32_t>();
    bool ordered = false;
    if (!plain && o.heavy_first && m->cost_K == K && (int32_t)m->cost.size() == nv && nsrc > 0) {
        // The heaviest sources, two per lane, go first (they would otherwise
        // set the tail); the rest keep vertex order, so that the sources in
        // flight together stay neighbours on the mesh and share its lines in L2
        // (full heaviest-first order is 3 % slower on the 750K torus, vertex
        // order 13 % slower on the 72.9K height field).
        std::vector<int32_t> ord((size_t)nsrc);
        for (int32_t i = 0; i < nsrc; ++i) ord[(size_t)i] = sb + i;
        const int64_t head = std::min<int64_t>(nsrc, (int64_t)lay.lanes * o.heavy_waves);
        std::vector<int32_t> byc(ord);
        std::stable_sort(byc.begin(), byc.end(),
                         [&](int32_t a, int32_t b) { return m->cost[(size_t)a] > m->cost[(size_t)b]; });
        std::vector<char> taken((size_t)nsrc, 0);
        for (int64_t i = 0; i < head; ++i) {
            ord[(size_t)i] = byc[(size_t)i];
            taken[(size_t)(byc[(size_t)i] - sb)] = 1;
        }
        int64_t k = head;
        for (int32_t i = 0; i < nsrc; ++i)
            if (!taken[(size_t)i]) ord[(size_t)k++] = sb + i;
        // The heaviest sources set the build's tail: one lane runs a source's
        // windows strictly one after another.  The cooperative warps run the
        // sources whose cost exceeds a lane's average share of the whole build
        // (the rest of the lanes finish about then), a whole warp each, with
        // fewer and shorter memory round trips per window.
        // The automatic share needs the costs of a build at this K: a K/10 probe
        // ranks the heaviest sources poorly (on the 72.9K height field its top
        // 200 hold 27 of K=500's top 200), and the tail adoption covers them.
        if (o.coop_sources > 0 || (o.coop_sources < 0 && !m->cost_probe)) {
            double total = 0.0;
            for (int32_t i = 0; i < nsrc; ++i) total += (double)m->cost[(size_t)(sb + i)];
            const double share = total / (double)lay.lanes;
            int64_t n = 0;
            if (o.coop_sources > 0) {
                n = std::min<int64_t>(o.coop_sources, nsrc);
            } else {
                while (n < head && (double)m->cost[(size_t)ord[(size_t)n]] >= share) ++n;
                n = std::min<int64_t>(n, lay.lanes / 64);
            }
            const int64_t warps = (int64_t)lay.lanes / 32;
            coop_n = (int32_t)n;
            // one cooperative warp per block at most (warp 0, whose block holds its heaps)
            coop_warps = (int32_t)std::min<int64_t>(
                {o.coop_warps > 0 ? (int64_t)o.coop_warps : std::max<int64_t>(1, n / 2), n, warps / 2,
                 (int64_t)lay.lanes / tpb});
            if (coop_warps <= 0) coop_n = 0;
        }
        SVG_CUDA(cudaMemcpyAsync(d_order, ord.data(), sizeof(int32_t) * (size_t)nsrc, cudaMemcpyHostToDevice, st));
        SVG_CUDA(cudaStreamSynchronize(st));
        ordered = true;
    }
    if (nsrc > 0 && !ordered) k_iota<<<(nsrc + 255) / 256, 256, 0, st>>>(d_order, nsrc, sb);
    // misc: work, retry_n, acc[8], cand_used ; retry list ; cand_n ; deg
    // retry list: room for the first pass's failures and, after them, the retry pass's
    size_t retry_bytes = align_up(sizeof(int32_t) * 2 * (size_t)std::max(nsrc, 1));
    size_t misc_bytes = 256 + retry_bytes + 2 * align_up(sizeof(int32_t) * ((size_t)nv + 1));
    b_misc.reserve(misc_bytes);
    SVG_CUDA(cudaMemsetAsync(b_misc.p, 0, misc_bytes, st));
    char* mp = b_misc.as<char>();
    int32_t* d_work = reinterpret_cast<int32_t*>(mp);
    int32_t* d_retry_n = d_work + 1;
    unsigned long long* d_acc = reinterpret_cast<unsigned long long*>(mp + 64);
    unsigned long long* d_cand_used = d_acc + 8;
    int32_t* d_retry = reinterpret_cast<int32_t*>(mp + 256);
    int32_t* d_cand_n = reinterpret_cast<int32_t*>(mp + 256 + retry_bytes);
    int32_t* d_deg = d_cand_n + align_up(sizeof(int32_t) * ((size_t)nv + 1)) / sizeof(int32_t);

    g->nv = nv;
    g->K = K;
    g->with_paths = o.with_paths != 0;
    g->st_windows = dev_alloc_n<int32_t>((size_t)nv * 3);
    g->st_maxq = g->st_windows + nv;
    g->st_flags = g->st_maxq + nv;
    SVG_CUDA(cudaMemsetAsync(g->st_windows, 0, sizeof(int32_t) * (size_t)nv * 3, st));
    g->off = dev_alloc_n<int64_t>((size_t)nv + 1);

    PhaseOut O{};
    O.order = d_order;
    O.nsrc = nsrc;
    O.work = d_work;
    O.retry = d_retry;
    O.retry_n = d_retry_n;
    O.cand_used = d_cand_used;
    O.cand_n = d_cand_n;
    O.deg = d_deg;
    O.st_windows = g->st_windows;
    O.st_maxq = g->st_maxq;
    O.st_flags = g->st_flags;
    O.acc = d_acc;
    O.coop_n = coop_n;
    O.coop_warps = coop_warps;
    O.coop_work = d_work + 4;
    O.coop_tail = o.coop_tail != 0 ? 1 : 0;

    cudaEvent_t ev[4];
    for (auto& e : ev) SVG_CUDA(cudaEventCreate(&e));
    int launches = 1;  // iota
    SVG_CUDA(cudaEventRecord(ev[0], st));

    DevBuf b_padj, b_pdist, b_ppath, b_tails;
    int32_t retry_n = 0;
    int32_t retry_host_cap_log2_v = lay.vcap_log2 + 1, retry_host_cap_log2_s = lay.scap_log2 + 2;
    int32_t smax_vlimit = lay.vlimit;
    int64_t scratch_bytes = (int64_t)(lane_bytes(lay) * lay.lanes);

    if (plain) {
        b_tails.reserve(sizeof(int32_t) * (size_t)std::max(nsrc, 1));
        b_padj.reserve(sizeof(int32_t) * (size_t)std::max(nsrc, 1) * K);
        b_pdist.reserve(sizeof(double) * (size_t)std::max(nsrc, 1) * K);
        if (g->with_paths) b_ppath.reserve(sizeof(PathEnd) * (size_t)std::max(nsrc, 1) * K);
        PlainOut P{};
        P.order = d_order;
        P.nsrc = nsrc;
        P.tails = b_tails.as<int32_t>();
        P.adj = b_padj.as<int32_t>();
        P.dist = b_pdist.as<double>();
        P.path = g->with_paths ? b_ppath.as<PathEnd>() : nullptr;
        P.stats = O;
        k_ich_plain<<<blocks, tpb, 0, st>>>(C, P);
        ++launches;
        SVG_CUDA(cudaGetLastError());
        SVG_CUDA(cudaMemcpyAsync(&retry_n, d_retry_n, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
        SVG_CUDA(cudaStreamSynchronize(st));
        if (retry_n > 0)
            throw SvgError{SVG_ERR_NOMEM, "plain build: a source outgrew its hash tables (raise K-based sizes)"};
    } else {
        int64_t cap = (int64_t)std::max(nsrc, 1) * ((int64_t)K + 64);
        for (int attempt = 0;; ++attempt) {
            b_cand.reserve(sizeof(Cand) * (size_t)cap);
            b_candstart.reserve(sizeof(int64_t) * ((size_t)nv + 1));
            O.cand = b_cand.as<Cand>();
            O.cand_cap = cap;
            O.cand_start = b_candstart.as<int64_t>();
            // the cooperative warps' heaps: window then pseudo-source entries
            const size_t coop_smem =
                coop_warps > 0 ? ((size_t)C.wstride * sizeof(WinEntry) + (size_t)C.pstride * sizeof(PsEntry)) : 0;
            if (coop_smem > 48 * 1024)
                SVG_CUDA(cudaFuncSetAttribute(k_ich_batched, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)coop_smem));
            k_ich_batched<<<blocks, tpb, coop_smem, st>>>(C, O);
            ++launches;
            cap_coop_smem = coop_smem;
            cap_pool = cap;
            cap_attempts = attempt;
            SVG_CUDA(cudaGetLastError());
            SVG_CUDA(cudaMemcpyAsync(&retry_n, d_retry_n, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
            unsigned long long used = 0;
            SVG_CUDA(cudaMemcpyAsync(&used, d_cand_used, sizeof(used), cudaMemcpyDeviceToHost, st));
            SVG_CUDA(cudaStreamSynchronize(st));
            if (retry_n > 0) {
                // Sources whose tables filled: rerun them with 2x vertex and 4x split tables.
                LaneConfig C2 = C;
                C2.wphys = C.wcap;
                C2.pphys = C.pcap;
                C2.wstride = heap_stride(C2.wphys);
                C2.pstride = heap_stride(C2.pphys);
                Layout l2 = lay;
                l2.wphys = C2.wphys;
                l2.pphys = C2.pphys;
                l2.vcap_log2 = retry_host_cap_log2_v;
                l2.scap_log2 = retry_host_cap_log2_s;
                l2.vlimit = (int32_t)(((int64_t)3 << l2.vcap_log2) / 4);
                C2.vcap_log2 = l2.vcap_log2;
                C2.scap_log2 = l2.scap_log2;
                C2.vlimit = l2.vlimit;
                C2.slimit = (int32_t)(((int64_t)3 << l2.scap_log2) / 4);
                int tb2 = 64;
                int bl2 = (int)std::min<int64_t>((retry_n + tb2 - 1) / tb2, (int64_t)prop.multiProcessorCount * 4);
                l2.lanes = bl2 * tb2;
                while (l2.lanes > 32 && (int64_t)(lane_bytes(l2) * l2.lanes) > budget) {
                    bl2 = std::max(1, bl2 / 2);
                    l2.lanes = bl2 * tb2;
                }
                carve(g_arena[1], l2, C2, st);
                scratch_bytes += (int64_t)(lane_bytes(l2) * l2.lanes);
                PhaseOut O2 = O;
                O2.coop_n = 0;
                O2.coop_warps = 0;
                O2.order = d_retry;
                O2.nsrc = retry_n;
                O2.work = d_work + 2;  // fresh queue head
                O2.retry = d_retry + retry_n;  // a second failure lands after the first list
                O2.retry_n = d_work + 3;
                SVG_CUDA(cudaMemsetAsync(d_work + 2, 0, 2 * sizeof(int32_t), st));
                k_ich_batched<<<bl2, tb2, 0, st>>>(C2, O2);
                ++launches;
                SVG_CUDA(cudaGetLastError());
                int32_t again = 0;
                SVG_CUDA(cudaMemcpyAsync(&again, d_work + 3, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
                SVG_CUDA(cudaMemcpyAsync(&used, d_cand_used, sizeof(used), cudaMemcpyDeviceToHost, st));
                SVG_CUDA(cudaStreamSynchronize(st));
                if (again > 0)
                    throw SvgError{SVG_ERR_NOMEM, "a source outgrew the enlarged retry tables"};
                smax_vlimit = std::max(smax_vlimit, l2.vlimit);
            }
            if ((int64_t)used <= cap) break;
            if (attempt >= 2) throw SvgError{SVG_ERR_NOMEM, "candidate pool kept overflowing"};
            cap = (int64_t)((double)used * 1.25) + 1024;
            SVG_CUDA(cudaMemsetAsync(b_misc.p, 0, misc_bytes, st));
            SVG_CUDA(cudaMemsetAsync(g->st_windows, 0, sizeof(int32_t) * (size_t)nv * 3, st));
        }
    }
    SVG_CUDA(cudaEventRecord(ev[1], st));

    // offsets = exclusive scan of degrees (vertices outside the range have 0)
    size_t tmp_bytes = 0;
    SVG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, d_deg, g->off, nv + 1, st));
    DevBuf b_tmp;
    b_tmp.reserve(tmp_bytes + 16);
    // d_deg[nv] is zero: the scan over nv+1 entries leaves the edge total in off[nv]
    SVG_CUDA(cub::DeviceScan::ExclusiveSum(b_tmp.p, tmp_bytes, d_deg, g->off, nv + 1, st));
    ++launches;
    int64_t nnz = 0;
    SVG_CUDA(cudaMemcpyAsync(&nnz, g->off + nv, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    SVG_CUDA(cudaStreamSynchronize(st));
    g->nnz = nnz;
    g->adj = dev_alloc_n<int32_t>((size_t)std::max<int64_t>(nnz, 1));
    g->dist = dev_alloc_n<double>((size_t)std::max<int64_t>(nnz, 1));
    if (g->with_paths) g->paths = dev_alloc(sizeof(PathEnd) * (size_t)std::max<int64_t>(nnz, 1));
    SVG_CUDA(cudaEventRecord(ev[2], st));

    if (plain) {
        k_compact<<<std::max(1, std::min(65535, (nsrc + 7) / 8)), 256, 0, st>>>(
            d_order, nsrc, K, b_tails.as<int32_t>(), b_padj.as<int32_t>(), b_pdist.as<double>(),
            g->with_paths ? b_ppath.as<PathEnd>() : nullptr, g->off, g->adj, g->dist,
            reinterpret_cast<PathEnd*>(g->paths));
        ++launches;
    } else if (nsrc > 0) {
        EmitParams E{};
        E.M = C.M;
        E.K = K;
        E.nv = nv;
        E.order = d_order;
        E.nsrc = nsrc;
        E.cand = b_cand.as<Cand>();
        E.cand_start = b_candstart.as<int64_t>();
        E.cand_n = d_cand_n;
        E.off = g->off;
        E.adj = g->adj;
        E.dist = g->dist;
        E.path = reinterpret_cast<PathEnd*>(g->paths);
        E.st_flags = g->st_flags;
        int smax = 32;
        while (smax < smax_vlimit) smax <<= 1;
        E.smax = smax;
        int wpb = (int)std::max<int64_t>(1, std::min<int64_t>(8, (96 * 1024) / ((int64_t)smax * 8)));
        size_t smem = (size_t)wpb * smax * 8;
        SVG_CUDA(cudaFuncSetAttribute(k_emit, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int eb = (int)std::min<int64_t>((nsrc + wpb - 1) / wpb, (int64_t)prop.multiProcessorCount * 16);
        k_emit<<<eb, wpb * 32, smem, st>>>(E);
        ++launches;
        if (SVG_SPLIT_TRACE && g->with_paths && nnz > 0) {
            k_trace<<<trace_blocks(nnz), 256, 0, st>>>(C.M, E.path, nnz, g->st_flags);
            ++launches;
        }
        cap_eb = eb;
        cap_wpb = wpb;
        cap_emit_smem = smem;
    }
    SVG_CUDA(cudaGetLastError());
    SVG_CUDA(cudaEventRecord(ev[3], st));
    SVG_CUDA(cudaStreamSynchronize(st));

    unsigned long long acc[8] = {0};
    SVG_CUDA(cudaMemcpy(acc, d_acc, sizeof(acc), cudaMemcpyDeviceToHost));
    float t01 = 0, t23 = 0, t03 = 0;
    SVG_CUDA(cudaEventElapsedTime(&t01, ev[0], ev[1]));
    SVG_CUDA(cudaEventElapsedTime(&t23, ev[2], ev[3]));
    SVG_CUDA(cudaEventElapsedTime(&t03, ev[0], ev[3]));
    for (auto& e : ev) cudaEventDestroy(e);

    svg_build_stats& S = g->stats;
    S = svg_build_stats{};
    S.ms_ich = t01;
    S.ms_emit = t23;
    S.ms_total = t01 + t23;  // excludes the host-side CSR allocation between the phases
    S.windows = (int64_t)acc[0];
    S.windows_generated = (int64_t)acc[1];
    S.pseudo_sources = (int64_t)acc[2];
    S.max_win_queue = (int32_t)acc[3];
    S.max_pseudo_queue = (int32_t)acc[4];
    S.edges = nnz;
    S.sources = nsrc;
    S.retried_sources = retry_n;
    S.launches = launches;
    S.scratch_bytes = scratch_bytes;
    S.coop_sources = coop_n;
    S.coop_warps = coop_warps;
    (void)t03;
    record_counts(m, g, K, sb, se, plain);
    if (o.graph && !plain && nsrc > 0 && retry_n == 0 && cap_attempts == 0) {
        CapturePlan P;
        P.C = C;
        P.O = O;
        P.blocks = blocks;
        P.tpb = tpb;
        P.coop_smem = cap_coop_smem;
        P.d_order = d_order;
        P.nsrc = nsrc;
        P.nv = nv;
        P.sb = sb;
        P.se = se;
        P.cap = cap_pool;
        P.nnz = nnz;
        P.tmp_bytes = tmp_bytes;
        P.misc_bytes = misc_bytes;
        P.retry_bytes = retry_bytes;
        P.eb = cap_eb;
        P.wpb = cap_wpb;
        P.emit_smem = cap_emit_smem;
        P.smax = 32;
        while (P.smax < smax_vlimit) P.smax <<= 1;
        P.with_paths = g->with_paths;
        P.lay = lay;
        P.scratch_bytes = scratch_bytes;
        P.coop_n = coop_n;
        P.coop_warps = coop_warps;
        capture_graph(m, o, P, g);
    }
    return SVG_OK;
}

// ------------------------------------------------------------ autotuner

namespace {
__device__ __forceinline__ unsigned long long mix64(unsigned long long x) {
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdULL;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ULL;
    x ^= x >> 33;
    return x;
}
// Order-independent checksum of a CSR: the sum of a mix of every (row, edge
// position, neighbour, length bits); equal graphs give equal sums.
__global__ void k_csr_checksum(const int64_t* off, const int32_t* adj, const double* dist, int32_t nv,
                               unsigned long long* out) {
    unsigned long long acc = 0;
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nv; v += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = off[v], e = off[v + 1];
        acc += mix64(((unsigned long long)v << 20) ^ (unsigned long long)(e - b));
        for (int64_t i = b; i < e; ++i)
            acc += mix64(((unsigned long long)(uint32_t)adj[i] << 32 | (unsigned long long)(i - b)) ^
                         mix64((unsigned long long)__double_as_longlong(dist[i])));
    }
    atomicAdd(out, acc);
}

unsigned long long csr_checksum(const svg_graph* g) {
    cudaStream_t st = lib_stream();
    unsigned long long* d = dev_alloc_n<unsigned long long>(1);
    SVG_CUDA(cudaMemsetAsync(d, 0, sizeof(*d), st));
    k_csr_checksum<<<256, 256, 0, st>>>(g->off, g->adj, g->dist, g->nv, d);
    SVG_CUDA(cudaGetLastError());
    unsigned long long h = 0;
    SVG_CUDA(cudaMemcpyAsync(&h, d, sizeof(h), cudaMemcpyDeviceToHost, st));
    SVG_CUDA(cudaStreamSynchronize(st));
    dev_free(d);
    return h;
}
}  // namespace

// Coordinate descent over the batched build's schedule parameters, each
// candidate timed as a full build (device time, CUDA events): the
// cooperative share (how many of the heaviest sources run on whole warps,
// then with how many warps), blocks per SM, the vote wait limit, the
// heavy-first waves and the physical heap factor.  A candidate replaces the
// best only when at least 2 % faster (one timing each).  Every candidate
// must build the graph of the first (checksum), else the tuner fails.
svg_status run_autotune(svg_mesh* m, const svg_build_opts& in, int32_t max_trials, svg_build_opts* out,
                        double* out_ms) {
    if (in.mode == SVG_BUILD_PLAIN) throw SvgError{SVG_ERR_ARG, "the autotuner tunes the batched build"};
    if (max_trials <= 0) max_trials = 16;
    svg_build_opts base = in;
    base.autotune = 0;
    if (base.heavy_first == 0) base.heavy_first = 1;
    base.coop_sources = 0;
    base.coop_warps = 0;
    base.coop_tail = 1;
    base.vote_wait = 8;
    base.heavy_waves = 2;
    base.heap_factor = 3;
    base.blocks = 0;
    int trials = 0;
    unsigned long long ref_sum = 0;
    bool have_ref = false;
    svg_build_stats last{};
    auto trial = [&](const svg_build_opts& o) -> double {
        svg_graph g;
        g.mesh = m;
        try {
            run_build(m, o, &g);
            const unsigned long long h = csr_checksum(&g);
            if (have_ref && h != ref_sum) throw SvgError{SVG_ERR_STATE, "autotune: a candidate built a different graph"};
            ref_sum = h;
            have_ref = true;
        } catch (...) {
            free_graph_device(&g);
            throw;
        }
        last = g.stats;
        free_graph_device(&g);
        ++trials;
        return last.ms_total;
    };
    trial(base);                   // records the per-source costs at this K (the work order)
    double best_ms = trial(base);  // the defaults, timed with that order
    svg_build_opts best = base;
    auto consider = [&](const svg_build_opts& o) {
        if (trials >= max_trials) return;
        const double ms = trial(o);
        if (ms < 0.98 * best_ms) {
            best_ms = ms;
            best = o;
        }
    };
    // threads per source: the heaviest sources on whole warps, the automatic
    // count (sources above a lane's average share) and half and twice it
    {
        svg_build_opts o = best;
        o.coop_sources = -1;
        consider(o);
    }
    const int32_t n_auto = last.coop_sources;
    for (int32_t n : {n_auto / 2, n_auto * 2}) {
        if (n <= 0) continue;
        svg_build_opts o = best;
        o.coop_sources = n;
        o.coop_warps = std::max(1, n / 2);
        consider(o);
    }
    if (best.coop_sources != 0) {
        const int32_t n = best.coop_sources > 0 ? best.coop_sources : n_auto;
        if (n > 0)
            for (int32_t w : {std::max(1, n / 4), n}) {
                svg_build_opts o = best;
                o.coop_sources = n;
                o.coop_warps = w;
                consider(o);
            }
    }
    // occupancy: one block of lanes per SM fewer than fit
    {
        int per_sm = 0, dev = 0, sms = 0;
        SVG_CUDA(cudaGetDevice(&dev));
        SVG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        SVG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_ich_batched, 128, 0));
        if (per_sm > 1) {
            svg_build_opts o = best;
            o.blocks = (per_sm - 1) * sms;
            consider(o);
        }
    }
    for (int32_t w : {4, 16}) {
        svg_build_opts o = best;
        o.vote_wait = w;
        consider(o);
    }
    for (int32_t w : {1, 4}) {
        svg_build_opts o = best;
        o.heavy_waves = w;
        consider(o);
    }
    for (int32_t f : {2, 4}) {
        svg_build_opts o = best;
        o.heap_factor = f;
        consider(o);
    }
    {  // the drained-queue adoption off
        svg_build_opts o = best;
        o.coop_tail = 0;
        consider(o);
    }
    bool found = false;
    for (auto& t : m->tuned)
        if (t.K == in.K) {
            t.opts = best;
            t.ms = best_ms;
            found = true;
        }
    if (!found) m->tuned.push_back({in.K, best, best_ms});
    if (out) {
        *out = best;
        out->autotune = 1;
    }
    if (out_ms) *out_ms = best_ms;
    return SVG_OK;
}

}  // namespace svgb

// ---------------------------------------------------------------------------
// Allocation-free build entry point (svg_build_rows_static).
//
// For callers that must not allocate device memory themselves or through the
// library - e.g. code running inside a framework that owns every allocation
// through its own pool, or a process that captures work into a graph whose
// memory must not change - this variant of the plain build keeps all of its
// lane scratch in one fixed array linked into the library, and writes into
// output buffers the caller provides.
//
// Limits: kStaticLanes = 128 lanes (one source each at a time, grid-stride
// over the range), K <= kStaticMaxK = 128, queue capacities fixed at the
// reference's 1023, tables sized as the regular build's first pass sizes them
// at K = 128 (2,048 vertex slots taking 1,536 keys, 2,048 split slots taking
// 1,536 keys).  The array takes kStaticScratchBytes (about 29 MiB) on every GPU
// that loads the library, for as long as the library stays loaded.  All calls
// share it: two calls whose kernels overlap on the GPU (different streams, or
// different host threads) race on it and produce garbage; serialise them.
// Each source resets its own tables before it starts, so nothing carried over
// from an earlier call is ever read and the array never needs clearing.
// ---------------------------------------------------------------------------
namespace svgb {
namespace {

constexpr int kStaticLanes = 128;
constexpr int kStaticMaxK = 128;
constexpr int kStaticWcap = 1023;
constexpr int kStaticPcap = 1023;
// The regular build's first-pass sizing at K = 128: vertex slots
// 2^(ceil(log2(2 * (2K + 1))) + SVG_TABLE_SHIFT) = 2048, split slots
// 2^(ceil(log2(8K)) + SVG_SPLIT_SHIFT) = 2048 (split keys reach about 1.6x the
// vertices reached), each filled to 3/4 at most.
constexpr int kStaticVcapLog2 = 10 + SVG_TABLE_SHIFT;
constexpr int kStaticScapLog2 = 10 + SVG_SPLIT_SHIFT;
constexpr int kStaticVlimit = (3 << kStaticVcapLog2) / 4;
constexpr int kStaticSlimit = (3 << kStaticScapLog2) / 4;

constexpr size_t al256(size_t x) { return (x + 255) / 256 * 256; }
constexpr int kStaticStride = (kStaticWcap + 16 + 3) / 4 * 4;  // heap entries per lane
constexpr size_t kSzWheap = al256((size_t)kStaticLanes * kStaticStride * sizeof(WinEntry));
constexpr size_t kSzWpool = al256((size_t)kStaticLanes * kStaticWcap * sizeof(WinPay));
constexpr size_t kSzWfree = al256((size_t)kStaticLanes * kStaticWcap * sizeof(uint16_t));
constexpr size_t kSzPheap = al256((size_t)kStaticLanes * kStaticStride * sizeof(PsEntry));
constexpr size_t kSzVtab = al256((size_t)kStaticLanes * ((size_t)1 << kStaticVcapLog2) * sizeof(VSlot));
constexpr size_t kSzVlist = al256((size_t)kStaticLanes * kStaticVlimit * sizeof(int32_t));
constexpr size_t kSzStab = al256((size_t)kStaticLanes * ((size_t)1 << kStaticScapLog2) * sizeof(SSlot));
constexpr size_t kSzEpoch = al256((size_t)kStaticLanes * sizeof(uint32_t));
constexpr size_t kStaticScratchBytes =
    kSzWheap + kSzWpool + kSzWfree + kSzPheap + kSzVtab + kSzVlist + kSzStab + kSzEpoch;

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

// Device address of g_static_scratch on the current device.  In host code the
// array's name is only a host-side stand-in for the symbol, never a device
// address.  The lookup runs on every call (it allocates nothing and costs
// microseconds), so a context re-created after cudaDeviceReset, which loads
// the module and its array anew, is never handed a stale address.  On a
// device's first call it also loads the library's kernels there.
void* static_scratch_address() {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess || p == nullptr) {
        cudaGetLastError();
        throw SvgError{SVG_ERR_CUDA, std::string("cudaGetSymbolAddress(static scratch) failed: ") +
                                         cudaGetErrorString(e)};
    }
    return p;
}

struct StaticOut {
    int32_t source_begin;
    int32_t nsrc;
    int32_t* tails;
    int32_t* adj;
    double* dist;
};

// The plain build (k_ich_plain) with its scratch carved from the static array.
// Row codes in tails: -1 the source outgrew the fixed tables; -2 an iteration
// cap stopped it or it reached a step the reference leaves undefined (the
// regular build reports both through its per-source flags).
__global__ void __launch_bounds__(128) k_ich_static(LaneConfig C, StaticOut O) {
    int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    int stride = gridDim.x * blockDim.x;
    Lane L(C, gtid);
    const int K = C.K;
    for (int r = gtid; r < O.nsrc; r += stride) {
        int v = O.source_begin + r;
        L.begin(v, true);
        while (!L.step()) {
        }
        int tail = 0;
        size_t row = (size_t)r * K;
        if (L.flags & kFlagCapacity) {
            O.tails[r] = -1;  // the source outgrew the static tables
            continue;
        }
        if (L.flags & (kFlagWatchdog | kFlagUndefined)) {
            O.tails[r] = -2;
            continue;
        }
        for (int j = 0; j < C.M.nv && K > 0; ++j) {
            double d = L.vdist(j);
            if (d == DBL_MAX || j == v) continue;
            uint32_t se, de;
            double sx = 0.0, dx = 0.0;
            if (trace_full(L, j, se, sx, de, dx)) continue;
            O.adj[row + tail] = j;
            O.dist[row + tail] = d;
            if (++tail == K) break;
        }
        // a back-trace can hit an iteration cap or an undefined step too
        O.tails[r] = (L.flags & (kFlagWatchdog | kFlagUndefined)) ? -2 : tail;
    }
}

}  // namespace
}  // namespace svgb

extern "C" svg_status svg_build_rows_static(svg_mesh* m, int32_t K, int32_t source_begin, int32_t source_end,
                                            int32_t* d_tails, int32_t* d_adj, double* d_dist, void* stream) {
    using namespace svgb;
    try {
        set_error("");
        if (!m || !d_tails || !d_adj || !d_dist) throw SvgError{SVG_ERR_ARG, "null argument"};
        if (!m->d.uploaded)
            throw SvgError{SVG_ERR_STATE, "mesh not on the device: call svg_mesh_upload first (it allocates)"};
        if (K < 1 || K > kStaticMaxK)
            throw SvgError{SVG_ERR_ARG, "K = " + std::to_string(K) + " outside [1, " + std::to_string(kStaticMaxK) +
                                            "], the limit of the allocation-free build"};
        if (source_begin < 0 || source_end > m->h.nv || source_begin > source_end)
            throw SvgError{SVG_ERR_ARG, "source range outside [0, nv]"};
        const int32_t nsrc = source_end - source_begin;
        if (nsrc == 0) return SVG_OK;
        char* base = static_cast<char*>(static_scratch_address());
        LaneConfig C{};
        C.M = m->d.view();
        C.K = K;
        C.wcap = kStaticWcap;
        C.pcap = kStaticPcap;
        C.wphys = kStaticWcap;
        C.pphys = kStaticPcap;
        C.wstride = kStaticStride;
        C.pstride = kStaticStride;
        C.vref = (uint32_t)K * 2;
        C.sref = (uint32_t)K * 10;
        C.vcap_log2 = kStaticVcapLog2;
        C.scap_log2 = kStaticScapLog2;
        C.vlimit = kStaticVlimit;
        C.slimit = kStaticSlimit;
        C.watchdog = (int64_t)1 << 26;
        char* p = base;
        C.wheap = reinterpret_cast<WinEntry*>(p); p += kSzWheap;
        C.wpool = reinterpret_cast<WinPay*>(p); p += kSzWpool;
        C.wfree = reinterpret_cast<uint16_t*>(p); p += kSzWfree;
        C.pheap = reinterpret_cast<PsEntry*>(p); p += kSzPheap;
        C.vtab = reinterpret_cast<VSlot*>(p); p += kSzVtab;
        C.vlist = reinterpret_cast<int32_t*>(p); p += kSzVlist;
        C.stab = reinterpret_cast<SSlot*>(p); p += kSzStab;
        C.epochs = reinterpret_cast<uint32_t*>(p);
        StaticOut O{source_begin, nsrc, d_tails, d_adj, d_dist};
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        k_ich_static<<<kStaticLanes / 128, 128, 0, st>>>(C, O);
        SVG_CUDA(cudaGetLastError());
        return SVG_OK;
    } catch (const SvgError& e) {
        set_error(e.msg);
        return e.code;
    } catch (const CudaFail& e) {
        cudaGetLastError();
        set_error(std::string("CUDA error ") + cudaGetErrorString(e.err) + " in " + e.where);
        return SVG_ERR_CUDA;
    }
}
