// Device ICH engine: one K-limited Improved-Chen-Han window propagation per
// lane, the reference's algorithm (ICHDevice.cu) step for step.
//
// Arithmetic: every expression that decides a branch or produces an output
// is the reference's, in the reference's operation order; the library is
// compiled with --fmad=false so nothing is contracted into an FMA.  Values
// that depend only on the mesh (corner angles, unfolded apex positions) are
// precomputed on the host with the same formulas and read here.
//
// Per-lane state lives in global memory (L1/L2-cached), sized per lane:
//   window heap : 16-byte {key, psrc, slot|birth} entries, 1-based binary
//                 min-heap with the reference's sift rules
//                 (PriorityQueue.cuh:48-105), one contiguous array per lane:
//                 the children 2i, 2i+1 of a node share one 32-byte sector and
//                 its grandchildren 4i..4i+3 one 64-byte span, so a sift-down
//                 fetches two levels per dependent memory round trip;
//   window pool : 48-byte payloads addressed by slot, recycled via a stack;
//   pseudo heap : 16-byte {key, vert, level<<8|birth} entries, same heap;
//   vertex table: 32-byte slots, open addressing, epoch-stamped (no clears);
//   split table : 32-byte slots, same scheme;
//   vertex list : table slots in insertion order (the emission walks only these).
//
// Two forms of a lane, the same algorithm and arithmetic:
//   LaneT<false>  one thread runs one source (the batched kernel's lanes, the
//                 plain and allocation-free builds);
//   LaneT<true>   a whole warp runs one heavy source: every thread holds the
//                 same state and runs the same scalar code (stores of one
//                 value by all threads are one store), while the memory-bound
//                 parts use the 32 threads - a sift-up loads every ancestor in
//                 one round trip and decides by ballot, a sift-down loads the
//                 five levels below a node in one round trip, and table
//                 lookups probe 8 slots of up to 4 keys at once.  The heap and
//                 table contents and the order of every operation are those
//                 of the one-thread form, so the results are bit-identical.
#pragma once

#include <cfloat>
#include <cstdint>

#include "svg_internal.h"

#ifndef SVG_ICH_INLINE_STALE
#define SVG_ICH_INLINE_STALE 8
#endif
// 1: the one-thread sifts prefetch keys only and re-read the moved entries;
// 0: they prefetch whole entries (one L1 round trip fewer per move).  With the
// three-level sift-down below, keys only measured 1.3 % faster (the sift-up
// holds fewer registers)
#ifndef SVG_KEYS_ONLY_SIFT
#define SVG_KEYS_ONLY_SIFT 1
#endif
// keys-only sift-up: ancestors whose keys are read in one round trip
#ifndef SVG_UP_LEVELS
#define SVG_UP_LEVELS 4
#endif
// 1: the keys-only sift-up reads a further batch of ancestors' keys per round
// trip while the climb goes on (0: one level per round trip past the first batch)
#ifndef SVG_UP_BATCHES
#define SVG_UP_BATCHES 1
#endif
// keys-only sift-up: up to this many ancestors, the moved entries are read
// into registers together and then written; beyond it, one at a time
#ifndef SVG_UP_ARRAY
#define SVG_UP_ARRAY 4
#endif
// 1: the one-thread sift-down reads the keys of three levels per round trip
// (measured 2.6 % faster on the 72.9K height field at K = 500, 4 % on the
// 750K torus)
#ifndef SVG_SIFT3
#define SVG_SIFT3 1
#endif
// 1: the free pool slot on top of the lane's free list is kept in a register,
// so a push does not wait for the list read (measured 1-1.5 % faster)
#ifndef SVG_FREE_CACHE
#define SVG_FREE_CACHE 1
#endif
// 1: a lane's counters and its cached look at the heap tops live in shared
// memory (one slot per thread, structure of arrays) instead of registers
// (measured 3-4 % faster)
#ifndef SVG_SMEM_STATE
#define SVG_SMEM_STATE 1
#endif
// 1: propagate() inserts a missing vertex or split entry at the empty slot its
// lookup ended on (no second probe walk; measured 2-4.5 % faster)
#ifndef SVG_INSERT_AT
#define SVG_INSERT_AT 1
#endif
// 1: propagate() builds, tests and pushes one child window at a time through
// one copy of the code (fewer live registers; measured 10 % faster)
#ifndef SVG_SEQ_CHILD
#define SVG_SEQ_CHILD 1
#endif

namespace svgb {

constexpr double kRefPi = 3.141592653589793238;  // Geometry.cuh:18
constexpr double kRelErr = 1e-8;                  // ICHDevice.cuh:10

// per-source flags
enum : int32_t {
    kFlagQueueDrop = 1,     // a push found its queue full and was dropped (reference behaviour)
    kFlagRefOverflow = 2,   // the reference's fixed-size hash table would have overflowed
    kFlagWatchdog = 4,      // an iteration cap stopped a loop the reference could spin in
    kFlagUndefined = 8,     // a step the reference leaves undefined (edges[-1])
    kFlagCapacity = 16,     // this lane's tables filled: the source is re-run with bigger ones
};

struct alignas(16) WinEntry {
    double key;     // window minDist
    int32_t psrc;   // pseudo-source vertex
    uint32_t sb;    // pool slot (low 16 bits) | birth (bits 16..23)
};
struct alignas(16) WinPay {
    double b0, b1;  // interval on the half-edge
    double sx, sy;  // unfolded (pseudo-)source, FlatenedSrc (ICHDevice.cuh:41-49)
    double psd;     // pseudoSrcDist
    int32_t cross;  // twin of the window's half-edge: where it propagates (-1: boundary)
    int32_t level;
};
struct alignas(16) PsEntry {
    double key;     // pseudo-source distance
    int32_t vert;
    uint32_t lb;    // level << 8 | birth
};
struct alignas(32) VSlot {
    uint32_t key;
    uint32_t epoch;
    int32_t enter;  // enterEdge
    int32_t birth;  // char birthTime, sign-extended
    double dist;
    int32_t sslot;  // split-table slot of `enter` when the vertex was reached through a window, else -1
    int32_t pad;
};
struct alignas(32) SSlot {
    uint32_t key;
    uint32_t epoch;
    int32_t psrc;   // pseudoSrcId
    int32_t pad;
    double dist;
    double x;
};

// A direct SVG candidate produced by the propagation phase.
struct alignas(8) Cand {
    int32_t u;      // vertex
    int32_t ee;     // enterEdge (edge key point), -1 = no interior key point
    double dist;
    double x;       // splitInfos[ee].x
};

// Path ends of an SVG edge (SVGNode fields other than adj/dist).
struct alignas(8) PathEnd {
    uint32_t src_edge, dst_edge;
    double src_x, dst_x;
};

struct LaneConfig {
    DevMesh M;
    int32_t K;
    int32_t wcap, pcap;      // logical queue capacities: pushes beyond them are dropped (reference)
    int32_t wphys, pphys;    // physical heap capacities (<= logical); exceeding one hands the
                             // source to the retry pass, which runs with physical = logical
    int32_t wstride, pstride;// heap entries per lane (>= phys + 16, multiple of 4)
    uint32_t vref, sref;     // the reference's table sizes, K*vert_coef and K*split_coef
    int32_t vcap_log2, scap_log2;
    int32_t vlimit, slimit;  // max keys this lane's tables take before kFlagCapacity
    int64_t watchdog;        // max steps per source
    int32_t max_wait;        // batched kernel: most iterations a lane waits for the vote to pick its step
    WinEntry* wheap;
    WinPay* wpool;
    uint16_t* wfree;
    PsEntry* pheap;
    VSlot* vtab;
    int32_t* vlist;
    SSlot* stab;
    uint32_t* epochs;
};

__device__ __forceinline__ int nxt(int e) { return (e % 3 == 2) ? e - 2 : e + 1; }
__device__ __forceinline__ int prv(int e) { return (e % 3 == 0) ? e + 2 : e - 1; }

__device__ __forceinline__ HeRec ld_he(const HeRec* p, int e) {
    const int4* q = reinterpret_cast<const int4*>(p + e);
    int4 a = __ldg(q);
    int4 b = __ldg(q + 1);
    HeRec h;
    h.v0 = a.x; h.v1 = a.y; h.twin = a.z; h.pad = a.w;
    h.len = __hiloint2double(b.y, b.x);
    h.corner = __hiloint2double(b.w, b.z);
    return h;
}
__device__ __forceinline__ double2 ld_apex(const HeGeo* g, int e) {
    return __ldg(reinterpret_cast<const double2*>(g + e));
}
__device__ __forceinline__ double2 ld_top(const HeGeo* g, int e) {
    return __ldg(reinterpret_cast<const double2*>(g + e) + 1);
}

// ICHDevice::Intersect (ICHDevice.cu:975-980)
__device__ __forceinline__ double isect(double v0x, double v0y, double v1x, double v1y, double p0x, double p0y,
                                        double p1x, double p1y) {
    double a00 = p0x - p1x, a01 = v1x - v0x, b0 = v1x - p1x;
    double a10 = p0y - p1y, a11 = v1y - v0y, b1 = v1y - p1y;
    return (b0 * a11 - b1 * a01) / (a00 * a11 - a10 * a01);
}
__device__ __forceinline__ double hyp(double x, double y) { return sqrt(x * x + y * y); }

// toLeft (Geometry.cu:306-310) with Vector2D::normalize (Geometry.cuh:35)
__device__ __forceinline__ bool to_left(double px, double py, double p0x, double p0y, double p1x, double p1y) {
    double ax = p1x - p0x, ay = p1y - p0y;
    double bx = px - p0x, by = py - p0y;
    double la = sqrt(ax * ax + ay * ay);
    if (!(fabs(la) < 1e-12)) { ax /= la; ay /= la; }
    double lb = sqrt(bx * bx + by * by);
    if (!(fabs(lb) < 1e-12)) { bx /= lb; by /= lb; }
    return (ax * by - ay * bx) > 0.0;
}

// A window being built: Window::calcMinDist + FlatenedSrc (ICHDevice.cuh:30-49)
// share xProj = (d0^2 + wLen^2 - d1^2) / (2 wLen).
struct NewWin {
    double key;
    WinPay p;
};
__device__ __forceinline__ void finish_window(double b0, double b1, double d0, double d1, double psd, NewWin& w) {
    double wLen = b1 - b0;
    double xProj = (d0 * d0 + wLen * wLen - d1 * d1) / (2 * wLen);
    double h = sqrt(fabs(d0 * d0 - xProj * xProj));
    if (xProj < 0.0) w.key = d0 + psd;
    else if (xProj > wLen) w.key = d1 + psd;
    else w.key = h + psd;
    w.p.b0 = b0;
    w.p.b1 = b1;
    w.p.sx = xProj + b0;
    w.p.sy = h;
    w.p.psd = psd;
}

// Group probe of up to four keys in 32-byte open-addressing slots (key at
// byte 0, epoch at byte 4): threads 8g..8g+7 walk key g's chain 8 slots per
// round, a ballot finds the first empty slot and any match before it (linear
// probing stops at the first empty slot, as the one-thread probes do).  Every
// thread of the warp calls it with the same arguments and receives the same
// results: slot (-1 if absent), the slot's two 16-byte halves, and the first
// empty slot of the chain (where an insert goes).
struct ProbeQ {
    const char* tbl;
    uint32_t mask;
    uint32_t h0;
    uint32_t key;
    bool on;
};
struct ProbeR {
    int slot;
    int empty;
    int4 head;
    int4 tail;
};
__device__ __forceinline__ void coop_probe4(const ProbeQ& q0, const ProbeQ& q1, const ProbeQ& q2, const ProbeQ& q3,
                                            uint32_t epoch, ProbeR& r0, ProbeR& r1, ProbeR& r2, ProbeR& r3) {
    constexpr unsigned kFull = 0xFFFFFFFFu;
    const int lane = threadIdx.x & 31, grp = lane >> 3, gl = lane & 7;
    // this thread's query, by value (a reference chosen by a thread-dependent
    // index would put the four queries in local memory)
    const char* q_tbl = grp == 0 ? q0.tbl : grp == 1 ? q1.tbl : grp == 2 ? q2.tbl : q3.tbl;
    const uint32_t q_mask = grp == 0 ? q0.mask : grp == 1 ? q1.mask : grp == 2 ? q2.mask : q3.mask;
    const uint32_t q_h0 = grp == 0 ? q0.h0 : grp == 1 ? q1.h0 : grp == 2 ? q2.h0 : q3.h0;
    const uint32_t q_key = grp == 0 ? q0.key : grp == 1 ? q1.key : grp == 2 ? q2.key : q3.key;
    r0.slot = r1.slot = r2.slot = r3.slot = -1;
    r0.empty = r1.empty = r2.empty = r3.empty = -1;
    unsigned open = (q0.on ? 0x000000FFu : 0u) | (q1.on ? 0x0000FF00u : 0u) | (q2.on ? 0x00FF0000u : 0u) |
                    (q3.on ? 0xFF000000u : 0u);
    for (uint32_t base = 0; open; base += 8) {
        const bool mine = (open >> lane) & 1u;
        const uint32_t h = (q_h0 + base + (uint32_t)gl) & q_mask;
        int4 hd = make_int4(0, 0, 0, 0), tl = hd;
        if (mine) {
            const int4* sp = reinterpret_cast<const int4*>(q_tbl + (size_t)h * 32);
            hd = sp[0];
            tl = sp[1];
        }
        const bool empty = mine && (uint32_t)hd.y != epoch;
        const bool hit = mine && !empty && (uint32_t)hd.x == q_key;
        const unsigned me = __ballot_sync(kFull, empty), mh = __ballot_sync(kFull, hit);
#pragma unroll
        for (int g = 0; g < 4; ++g) {
            ProbeR& r = g == 0 ? r0 : g == 1 ? r1 : g == 2 ? r2 : r3;
            const ProbeQ& qg = g == 0 ? q0 : g == 1 ? q1 : g == 2 ? q2 : q3;
            if (!((open >> (8 * g)) & 1u)) continue;
            const unsigned ge = (me >> (8 * g)) & 0xFFu, gh = (mh >> (8 * g)) & 0xFFu;
            const int fe = ge ? __ffs(ge) - 1 : 8;
            const unsigned hb = fe < 8 ? (gh & ((1u << fe) - 1u)) : gh;
            if (hb) {
                const int src = 8 * g + __ffs(hb) - 1;
                r.slot = (int)((qg.h0 + base + (uint32_t)(src - 8 * g)) & qg.mask);
                r.head.x = __shfl_sync(kFull, hd.x, src);
                r.head.y = __shfl_sync(kFull, hd.y, src);
                r.head.z = __shfl_sync(kFull, hd.z, src);
                r.head.w = __shfl_sync(kFull, hd.w, src);
                r.tail.x = __shfl_sync(kFull, tl.x, src);
                r.tail.y = __shfl_sync(kFull, tl.y, src);
                r.tail.z = __shfl_sync(kFull, tl.z, src);
                r.tail.w = __shfl_sync(kFull, tl.w, src);
                open &= ~(0xFFu << (8 * g));
            } else if (fe < 8) {
                r.empty = (int)((qg.h0 + base + (uint32_t)fe) & qg.mask);
                open &= ~(0xFFu << (8 * g));
            } else if (base > qg.mask) {  // a full table with no empty slot: absent, nowhere to insert
                open &= ~(0xFFu << (8 * g));
            }
        }
    }
}
__device__ __forceinline__ ProbeQ probe_q(const void* tbl, int log2cap, uint32_t key, bool on) {
    ProbeQ q;
    q.tbl = static_cast<const char*>(tbl);
    q.mask = (1u << log2cap) - 1u;
    q.h0 = (key * 0x9E3779B1u) >> (32 - log2cap);
    q.key = key;
    q.on = on;
    return q;
}
__device__ __forceinline__ ProbeQ probe_off() {
    ProbeQ q;
    q.tbl = nullptr;
    q.mask = 0;
    q.h0 = 0;
    q.key = 0;
    q.on = false;
    return q;
}

#if SVG_SMEM_STATE
// Per-thread slots (blocks of up to 128 threads) of the lane state that a
// step touches once or twice: counters and the cached heap tops.
struct LaneSmem {
    double wkey[128];
    int32_t wpsrc[128];
    uint32_t wsb[128];
    double pkey[128];
    int32_t pvert[128];
    uint32_t plb[128];
    int32_t windows[128], pseudos[128], generated[128], maxw[128], maxp[128];
    long long steps[128];
};
__shared__ LaneSmem g_lane_smem;
#endif

template <bool kCoop>
struct LaneT {
    const LaneConfig& C;
    // This lane's scratch, derived from its index when used (held pointers
    // would take fourteen registers for the whole loop).
    int32_t lid;
    // The cooperative form keeps its source's two heaps in shared memory
    // (sheap: wstride window entries, then pstride pseudo-source entries), or,
    // for a source it adopted from a lane (sheap null), in that lane's scratch.
    WinEntry* sheap = nullptr;
    __device__ __forceinline__ WinEntry* WH() const {
        if constexpr (kCoop)
            if (sheap) return sheap;
        return C.wheap + (size_t)lid * C.wstride;
    }
    __device__ __forceinline__ PsEntry* PH() const {
        if constexpr (kCoop)
            if (sheap) return reinterpret_cast<PsEntry*>(sheap + C.wstride);
        return C.pheap + (size_t)lid * C.pstride;
    }
    __device__ __forceinline__ WinPay* WP() const { return C.wpool + (size_t)lid * C.wphys; }
    __device__ __forceinline__ uint16_t* WF() const { return C.wfree + (size_t)lid * C.wphys; }
    __device__ __forceinline__ VSlot* VT() const { return C.vtab + ((size_t)lid << C.vcap_log2); }
    __device__ __forceinline__ int32_t* VL() const { return C.vlist + (size_t)lid * C.vlimit; }
    __device__ __forceinline__ SSlot* ST() const { return C.stab + ((size_t)lid << C.scap_log2); }
    int wsize, psize, nfree, nfresh;
    int ftop;       // WF()[nfree - 1] when nfree > 0 (free-slot cache)
    int vcount, scount;
    uint32_t epoch;
    int source;
    int src_birth;
    int total;      // totalCalcVertNum
    int flags;
#if SVG_SMEM_STATE
    __device__ __forceinline__ int& st_windows() const { return g_lane_smem.windows[threadIdx.x]; }
    __device__ __forceinline__ int& st_pseudos() const { return g_lane_smem.pseudos[threadIdx.x]; }
    __device__ __forceinline__ int& st_generated() const { return g_lane_smem.generated[threadIdx.x]; }
    __device__ __forceinline__ int& st_maxw() const { return g_lane_smem.maxw[threadIdx.x]; }
    __device__ __forceinline__ int& st_maxp() const { return g_lane_smem.maxp[threadIdx.x]; }
    __device__ __forceinline__ long long& st_steps() const { return g_lane_smem.steps[threadIdx.x]; }
#else
    int windows_, pseudos_, generated_, maxw_, maxp_;
    long long steps_;
    __device__ __forceinline__ int& st_windows() { return windows_; }
    __device__ __forceinline__ int& st_pseudos() { return pseudos_; }
    __device__ __forceinline__ int& st_generated() { return generated_; }
    __device__ __forceinline__ int& st_maxw() { return maxw_; }
    __device__ __forceinline__ int& st_maxp() { return maxp_; }
    __device__ __forceinline__ long long& st_steps() { return steps_; }
    __device__ __forceinline__ int st_windows() const { return windows_; }
    __device__ __forceinline__ int st_pseudos() const { return pseudos_; }
    __device__ __forceinline__ int st_generated() const { return generated_; }
    __device__ __forceinline__ int st_maxw() const { return maxw_; }
    __device__ __forceinline__ int st_maxp() const { return maxp_; }
    __device__ __forceinline__ long long st_steps() const { return steps_; }
#endif

    // gtid: the thread's global index (one-thread form) or the warp's first
    // thread's (cooperative form: the warp uses that thread's scratch).
    __device__ LaneT(const LaneConfig& c, int gtid) : C(c) {
        lid = gtid;
        epoch = C.epochs[gtid];
    }

    // Cooperative form: take over the source lane o of this warp is running
    // in the one-thread form (every thread calls it; the state comes from
    // lane o by shuffles, the scratch and heaps stay lane o's).  The adopted
    // source continues exactly where the lane stood: the next step re-reads
    // the heap tops the lane's cached look was taken from.
    template <class Other>
    __device__ void adopt(const Other& L, int o) {
        constexpr unsigned kFull = 0xFFFFFFFFu;
        sheap = nullptr;
        lid = __shfl_sync(kFull, L.lid, o);
        wsize = __shfl_sync(kFull, L.wsize, o);
        psize = __shfl_sync(kFull, L.psize, o);
        nfree = __shfl_sync(kFull, L.nfree, o);
        nfresh = __shfl_sync(kFull, L.nfresh, o);
        ftop = __shfl_sync(kFull, L.ftop, o);
        vcount = __shfl_sync(kFull, L.vcount, o);
        scount = __shfl_sync(kFull, L.scount, o);
        epoch = __shfl_sync(kFull, L.epoch, o);
        source = __shfl_sync(kFull, L.source, o);
        src_birth = __shfl_sync(kFull, L.src_birth, o);
        total = __shfl_sync(kFull, L.total, o);
        flags = __shfl_sync(kFull, L.flags, o);
        // (with SVG_SMEM_STATE both lanes' counters are this thread's slot:
        // each thread reads its slot, the shuffle syncs, each writes its slot)
        const int sw = __shfl_sync(kFull, L.st_windows(), o);
        const int sp = __shfl_sync(kFull, L.st_pseudos(), o);
        const int sg = __shfl_sync(kFull, L.st_generated(), o);
        const int smw = __shfl_sync(kFull, L.st_maxw(), o);
        const int smp = __shfl_sync(kFull, L.st_maxp(), o);
        const long long sst = __shfl_sync(kFull, L.st_steps(), o);
        st_windows() = sw;
        st_pseudos() = sp;
        st_generated() = sg;
        st_maxw() = smw;
        st_maxp() = smp;
        st_steps() = sst;
        done = __shfl_sync(kFull, (int)L.done, o) != 0;
        pk_valid = false;
    }

    __device__ __forceinline__ WinEntry& wh(int i) { return WH()[i]; }
    __device__ __forceinline__ PsEntry& ph(int i) { return PH()[i]; }

    // ---------------------------------------------------------- tables
    __device__ __forceinline__ uint32_t vhash(uint32_t k) const { return (k * 0x9E3779B1u) >> (32 - C.vcap_log2); }
    __device__ __forceinline__ uint32_t shash(uint32_t k) const { return (k * 0x9E3779B1u) >> (32 - C.scap_log2); }

    // One key's group probe (cooperative form).
    __device__ __forceinline__ ProbeR probe1(const void* tbl, int log2cap, uint32_t key) const {
        ProbeR r0, r1, r2, r3;
        coop_probe4(probe_q(tbl, log2cap, key, true), probe_off(), probe_off(), probe_off(), epoch, r0, r1, r2, r3);
        return r0;
    }

    // slot index of vertex v, or -1 if absent
    __device__ __forceinline__ int vfind(int v) {
        if constexpr (kCoop) return probe1(VT(), C.vcap_log2, (uint32_t)v).slot;
        uint32_t mask = (1u << C.vcap_log2) - 1, h = vhash((uint32_t)v);
        for (;;) {
            uint2 ke = *reinterpret_cast<const uint2*>(&VT()[h]);
            if (ke.y != epoch) return -1;
            if (ke.x == (uint32_t)v) return (int)h;
            h = (h + 1) & mask;
        }
    }
    // First probe of a lookup, issued without waiting: slot key/epoch/enter/birth
    // and the distance (one 32-byte sector).  vfinish completes the probe chain.
    __device__ __forceinline__ void vfirst(int v, uint32_t& h, int4& k, double& d) const {
        h = vhash((uint32_t)v);
        k = *reinterpret_cast<const int4*>(&VT()[h]);
        d = VT()[h].dist;
    }
    // h ends at the key's slot, or at the empty slot where an insert goes
    __device__ __forceinline__ int vfinish(int v, uint32_t& h, int4& k, double& d) const {
        const uint32_t mask = (1u << C.vcap_log2) - 1;
        for (;;) {
            if ((uint32_t)k.y != epoch) { d = DBL_MAX; return -1; }
            if ((uint32_t)k.x == (uint32_t)v) return (int)h;
            h = (h + 1) & mask;
            k = *reinterpret_cast<const int4*>(&VT()[h]);
            d = VT()[h].dist;
        }
    }
    __device__ __forceinline__ void sfirst(int e, uint32_t& h, int4& k, double2& dx) const {
        h = shash((uint32_t)e);
        k = *reinterpret_cast<const int4*>(&ST()[h]);
        dx = *reinterpret_cast<const double2*>(&ST()[h].dist);
    }
    // returns the slot or -1; dx = {dist, x} of the entry, {DBL_MAX, DBL_MAX} if absent
    __device__ __forceinline__ int sfinish(int e, uint32_t& h, int4& k, double2& dx) const {
        const uint32_t mask = (1u << C.scap_log2) - 1;
        for (;;) {
            if ((uint32_t)k.y != epoch) { dx.x = DBL_MAX; dx.y = DBL_MAX; return -1; }
            if ((uint32_t)k.x == (uint32_t)e) return (int)h;
            h = (h + 1) & mask;
            k = *reinterpret_cast<const int4*>(&ST()[h]);
            dx = *reinterpret_cast<const double2*>(&ST()[h].dist);
        }
    }
    __device__ __forceinline__ double vdist(int v) {
        int s = vfind(v);
        return s < 0 ? DBL_MAX : VT()[s].dist;
    }
    __device__ __forceinline__ int vbirth(int v) {
        int s = vfind(v);
        return s < 0 ? -1 : VT()[s].birth;
    }
    // MyHashTable::operator[] (MyHashTable.cuh:72-82): find or insert with defaults
    __device__ int vput(int v) {
        uint32_t h;
        if constexpr (kCoop) {
            const ProbeR r = probe1(VT(), C.vcap_log2, (uint32_t)v);
            if (r.slot >= 0) return r.slot;
            h = (uint32_t)r.empty;  // vlimit keeps a quarter of the slots empty: never -1
        } else {
            uint32_t mask = (1u << C.vcap_log2) - 1;
            h = vhash((uint32_t)v);
            for (;;) {
                uint2 ke = *reinterpret_cast<const uint2*>(&VT()[h]);
                if (ke.y != epoch) break;
                if (ke.x == (uint32_t)v) return (int)h;
                h = (h + 1) & mask;
            }
        }
        return vinsert(v, h);
    }
    // Insert vertex v at h, the empty slot that ends its probe chain.
    __device__ int vinsert(int v, uint32_t h) {
        if (vcount >= C.vlimit) {  // keep the probe chains short: hand the source to the big pass
            flags |= kFlagCapacity;
            return -1;
        }
        VSlot s;
        s.key = (uint32_t)v; s.epoch = epoch; s.enter = -1; s.birth = -1; s.dist = DBL_MAX; s.sslot = -1; s.pad = 0;
        VT()[h] = s;
        VL()[vcount] = (int32_t)h;
        ++vcount;
        if ((uint32_t)vcount > C.vref) flags |= kFlagRefOverflow;
        return (int)h;
    }
    __device__ __forceinline__ int sfind(int e) {
        if constexpr (kCoop) return probe1(ST(), C.scap_log2, (uint32_t)e).slot;
        uint32_t mask = (1u << C.scap_log2) - 1, h = shash((uint32_t)e);
        for (;;) {
            uint2 ke = *reinterpret_cast<const uint2*>(&ST()[h]);
            if (ke.y != epoch) return -1;
            if (ke.x == (uint32_t)e) return (int)h;
            h = (h + 1) & mask;
        }
    }
    __device__ int sput(int e) {
        uint32_t h;
        if constexpr (kCoop) {
            const ProbeR r = probe1(ST(), C.scap_log2, (uint32_t)e);
            if (r.slot >= 0) return r.slot;
            h = (uint32_t)r.empty;  // slimit keeps a quarter of the slots empty: never -1
        } else {
            uint32_t mask = (1u << C.scap_log2) - 1;
            h = shash((uint32_t)e);
            for (;;) {
                uint2 ke = *reinterpret_cast<const uint2*>(&ST()[h]);
                if (ke.y != epoch) break;
                if (ke.x == (uint32_t)e) return (int)h;
                h = (h + 1) & mask;
            }
        }
        return sinsert(e, h);
    }
    // Insert half-edge e at h, the empty slot that ends its probe chain.
    __device__ int sinsert(int e, uint32_t h) {
        if (scount >= C.slimit) {
            flags |= kFlagCapacity;
            return -1;
        }
        SSlot s;
        s.key = (uint32_t)e; s.epoch = epoch; s.psrc = -1; s.pad = 0; s.dist = DBL_MAX; s.x = DBL_MAX;
        ST()[h] = s;
        ++scount;
        if ((uint32_t)scount > C.sref) flags |= kFlagRefOverflow;
        return (int)h;
    }
    // Reset every slot (the plain build's per-source Clear, ICHDevice.cu:487-523).
    __device__ void clear_tables() {
        for (int i = 0; i < (1 << C.vcap_log2); ++i) {
            VSlot s;
            s.key = 0xFFFFFFFFu; s.epoch = 0; s.enter = -1; s.birth = -1; s.dist = DBL_MAX; s.sslot = -1; s.pad = 0;
            VT()[i] = s;
        }
        for (int i = 0; i < (1 << C.scap_log2); ++i) {
            SSlot s;
            s.key = 0xFFFFFFFFu; s.epoch = 0; s.psrc = -1; s.pad = 0; s.dist = DBL_MAX; s.x = DBL_MAX;
            ST()[i] = s;
        }
    }

    // ----------------------------------------------------------- heaps
    // The reference's sift-up (PriorityQueue.cuh:57-64): the new entry moves up
    // while its parent's key is greater.  On the benchmark mesh 69 % of the
    // window pushes do not move and 11.6 % climb past four levels.  Four
    // ancestors are loaded per round trip (they are what the level-by-level
    // loop would read: a move only writes below the next ancestor); the number
    // of moves over them is counted with the same stop rule and the moves are
    // written predicated, so no data-dependent branch splits the lanes; with
    // SVG_UP_BATCHES a longer climb takes the next four the same way, else it
    // continues level by level.
    template <class T>
    __device__ __forceinline__ int sift_up(T* H, int cur, const T& x) {
        if constexpr (kCoop) {
            // thread j holds ancestor cur >> (j + 1); the moves are the
            // ancestors, from the parent up, whose key exceeds x's
            const int lane = threadIdx.x & 31;
            const int a = lane < 30 ? (cur >> (lane + 1)) : 0;
            T e;
            e.key = 0.0;
            if (a > 0) e = H[a];
            const unsigned gt = __ballot_sync(0xFFFFFFFFu, a > 0 && e.key > x.key);
            const int m = __ffs(~gt) - 1;
            if (lane < m) H[cur >> lane] = e;
            H[cur >> m] = x;
            __syncwarp();
            return cur >> m;
        } else {
            constexpr int kUp = SVG_KEYS_ONLY_SIFT ? SVG_UP_LEVELS : 4;
#if SVG_KEYS_ONLY_SIFT && SVG_UP_BATCHES
            // batches of kUp ancestors' keys, one round trip each, for as long
            // as the climb goes on: the same stop rule level by level, since a
            // batch's moves only shift entries below its top ancestor (a
            // tenth of the pushes climb past four levels)
            int c = cur;
            for (;;) {
                double ak[kUp];
#pragma unroll
                for (int j = 0; j < kUp; ++j) ak[j] = (c >> (j + 1)) > 0 ? H[c >> (j + 1)].key : 0.0;
                int m = 0;
#pragma unroll
                for (int j = 0; j < kUp; ++j)
                    if (m == j && (c >> (j + 1)) > 0 && ak[j] > x.key) m = j + 1;
                if constexpr (kUp <= SVG_UP_ARRAY) {
                    T mv[kUp];
#pragma unroll
                    for (int j = 0; j < kUp; ++j)
                        if (j < m) mv[j] = H[c >> (j + 1)];
#pragma unroll
                    for (int j = 0; j < kUp; ++j)
                        if (j < m) H[c >> j] = mv[j];
                } else {
                    for (int j = 0; j < m; ++j) H[c >> j] = H[c >> (j + 1)];
                }
                c >>= m;
                if (m < kUp) break;
            }
            H[c] = x;
            return c;
#elif SVG_KEYS_ONLY_SIFT
            // keys of the first kUp ancestors in one round trip; the moved
            // entries are read again (their sectors were just fetched) before
            // each is written one level down
            double ak[kUp];
#pragma unroll
            for (int j = 0; j < kUp; ++j) ak[j] = (cur >> (j + 1)) > 0 ? H[cur >> (j + 1)].key : 0.0;
            int m = 0;
#pragma unroll
            for (int j = 0; j < kUp; ++j)
                if (m == j && (cur >> (j + 1)) > 0 && ak[j] > x.key) m = j + 1;
            if constexpr (kUp <= SVG_UP_ARRAY) {
                T mv[kUp];
#pragma unroll
                for (int j = 0; j < kUp; ++j)
                    if (j < m) mv[j] = H[cur >> (j + 1)];
#pragma unroll
                for (int j = 0; j < kUp; ++j)
                    if (j < m) H[cur >> j] = mv[j];
            } else {
                // one entry at a time, top-down reads after the writes below
                // them (each read hits the sector just fetched)
                for (int j = 0; j < m; ++j) H[cur >> j] = H[cur >> (j + 1)];
            }
#else
            // the first four ancestors in one round trip (they are what the level-
            // by-level loop would read: a move only writes below the next
            // ancestor); the moves over them are counted with the same stop rule
            // and written predicated
            T anc[4];
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if ((cur >> (j + 1)) > 0) anc[j] = H[cur >> (j + 1)];
            int m = 0;
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (m == j && (cur >> (j + 1)) > 0 && anc[j].key > x.key) m = j + 1;
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (j < m) H[cur >> j] = anc[j];
#endif
#if !(SVG_KEYS_ONLY_SIFT && SVG_UP_BATCHES)
            int c = cur >> m;
            if (m == kUp) {
                for (;;) {
                    const int p = c >> 1;
                    if (p == 0) break;
                    const T pe = H[p];
                    if (!(pe.key > x.key)) break;
                    H[c] = pe;
                    c = p;
                }
            }
            H[c] = x;
            return c;
#endif
        }
    }

    // Push (PriorityQueue.cuh:48-67).
    __device__ void wpush(const NewWin& w, int psrc, int birth) {
        ++st_generated();  // counts attempts, like numOfWinGen
        if (wsize >= C.wcap) {  // PriorityQueue.cuh:53: dropped when full
            flags |= kFlagQueueDrop;
            return;
        }
        if (wsize >= C.wphys) {  // beyond this lane's physical heap: retry with a full one
            flags |= kFlagCapacity;
            return;
        }
#if SVG_FREE_CACHE
        // the list entry under the cached top is loaded now and used by the
        // next push, after this push's sift-up
        int slot;
        if (nfree > 0) {
            slot = ftop;
            if (--nfree > 0) ftop = WF()[nfree - 1];
        } else {
            slot = nfresh++;
        }
#else
        const int slot = nfree > 0 ? (int)WF()[--nfree] : nfresh++;
#endif
        WP()[slot] = w.p;
        WinEntry e;
        e.key = w.key;
        e.psrc = psrc;
        e.sb = (uint32_t)slot | ((uint32_t)(birth & 0xFF) << 16);
        sift_up(WH(), ++wsize, e);
        if (wsize > st_maxw()) st_maxw() = wsize;
    }
    // Cooperative sift-down: the 62 nodes 1-5 levels below `cur` are loaded
    // in one round trip (two per thread: node k, k+32 of the subtree in level
    // order), the path is chosen level by level from shuffled keys with the
    // rules below, and each moved node is written by the thread holding it.
    // Every node is read before any write of that round, and a round writes
    // only nodes above the next round's subtree.
    template <class T>
    __device__ __forceinline__ int coop_sift_down(T* H, int n, const T& last) {
        constexpr unsigned kFull = 0xFFFFFFFFu;
        const int lane = threadIdx.x & 31;
        int cur = 1;
        for (int round = 0; round < 8; ++round) {
            if ((cur << 1) > n) break;
            T e[2];
#pragma unroll
            for (int r = 0; r < 2; ++r) {
                const int k = lane + 32 * r;       // subtree node in level order
                const int d = 31 - __clz(k + 2);   // its depth below cur (1..5)
                const int ix = k < 62 ? (cur << d) + (k + 2 - (1 << d)) : n + 1;
                e[r].key = 0.0;
                if (ix <= n) e[r] = H[ix];
            }
            int p = cur;
            bool moved_all = true;
#pragma unroll
            for (int d = 1; d <= 5; ++d) {
                const int l = p << 1;
                if (l > n) { moved_all = false; break; }
                const int kl = l - (cur << d) + (1 << d) - 2;  // subtree position of l (l + 1 is kl + 1)
                const double al = __shfl_sync(kFull, (kl >> 5) ? e[1].key : e[0].key, kl & 31);
                const double bl = __shfl_sync(kFull, ((kl + 1) >> 5) ? e[1].key : e[0].key, (kl + 1) & 31);
                const int k1 = (l + 1 <= n && !(al < bl)) ? 1 : 0;
                if (!((k1 ? bl : al) < last.key)) { moved_all = false; break; }
                const int kc = kl + k1;
                if (lane == (kc & 31)) H[p] = (kc >> 5) ? e[1] : e[0];
                p = l + k1;
            }
            cur = p;
            if (!moved_all) break;
        }
        __syncwarp();
        return cur;
    }

    // The reference's sift-down (PriorityQueue.cuh:76-105): the children of
    // `cur` are compared with each other (ties go right) and the smaller moves
    // up while it is smaller than the last element.  The keys of three levels
    // below `cur` (SVG_SIFT3; two without it) are loaded together, so those
    // levels cost one dependent round trip (reads past the heap's end stay
    // inside the lane's array, stride >= cap + 8, and are never used); the
    // moved entries are read again from the sectors just fetched and written
    // with predicated stores, one exit test per round trip.
    template <class T>
    __device__ __forceinline__ int sift_down2(T* H, int n, const T& last) {
        if constexpr (kCoop) return coop_sift_down(H, n, last);
        int cur = 1;
        for (;;) {
            const int l = cur << 1;
            if (l > n) break;
#if SVG_SIFT3
            // keys of three levels below cur (2 + 4 + 8) in one round trip
            // (reads past the heap's end stay inside the lane's array,
            // stride >= cap + 8, and are never used); the moved entries are
            // read again from the sectors just fetched
            const double a = H[l].key, b = H[l + 1].key;
            const int g = cur << 2, h8 = cur << 3;
            double q0 = 0.0, q1 = 0.0, q2 = 0.0, q3 = 0.0;
            if (g <= n) { q0 = H[g].key; q1 = H[g + 1].key; q2 = H[g + 2].key; q3 = H[g + 3].key; }
            double r0 = 0.0, r1 = 0.0, r2 = 0.0, r3 = 0.0, r4 = 0.0, r5 = 0.0, r6 = 0.0, r7 = 0.0;
            if (h8 <= n) {
                r0 = H[h8].key; r1 = H[h8 + 1].key; r2 = H[h8 + 2].key; r3 = H[h8 + 3].key;
                r4 = H[h8 + 4].key; r5 = H[h8 + 5].key; r6 = H[h8 + 6].key; r7 = H[h8 + 7].key;
            }
            const int k1 = (l + 1 <= n && !(a < b)) ? 1 : 0;
            const bool mv1 = (k1 ? b : a) < last.key;
            const int c1 = l + k1;
            const int l2 = c1 << 1;
            const double a2 = k1 ? q2 : q0, b2 = k1 ? q3 : q1;
            const int k2 = (l2 + 1 <= n && !(a2 < b2)) ? 1 : 0;
            const bool mv2 = mv1 && l2 <= n && (k2 ? b2 : a2) < last.key;
            const int c2 = l2 + k2;
            const int l3 = c2 << 1;  // = h8 + 4 k1 + 2 k2
            const double a3 = k1 ? (k2 ? r6 : r4) : (k2 ? r2 : r0);
            const double b3 = k1 ? (k2 ? r7 : r5) : (k2 ? r3 : r1);
            const int k3 = (l3 + 1 <= n && !(a3 < b3)) ? 1 : 0;
            const bool mv3 = mv2 && l3 <= n && (k3 ? b3 : a3) < last.key;
            const int c3 = l3 + k3;
            T e1, e2, e3;
            if (mv1) e1 = H[c1];
            if (mv2) e2 = H[c2];
            if (mv3) e3 = H[c3];
            if (mv1) H[cur] = e1;
            if (mv2) H[c1] = e2;
            if (mv3) H[c2] = e3;
            cur = mv3 ? c3 : (mv2 ? c2 : (mv1 ? c1 : cur));
            const bool more = mv3;
#elif SVG_KEYS_ONLY_SIFT
            const double a = H[l].key, b = H[l + 1].key;
            const int g = cur << 2;
            double q0 = 0.0, q1 = 0.0, q2 = 0.0, q3 = 0.0;
            if (g <= n) { q0 = H[g].key; q1 = H[g + 1].key; q2 = H[g + 2].key; q3 = H[g + 3].key; }
            const int k1 = (l + 1 <= n && !(a < b)) ? 1 : 0;
            const bool mv1 = (k1 ? b : a) < last.key;
            const int c1 = l + k1;
            const int l2 = c1 << 1;
            const double a2 = k1 ? q2 : q0, b2 = k1 ? q3 : q1;
            const int k2 = (l2 + 1 <= n && !(a2 < b2)) ? 1 : 0;
            const bool mv2 = mv1 && l2 <= n && (k2 ? b2 : a2) < last.key;
            const int c2 = l2 + k2;
            T e1, e2;
            if (mv1) e1 = H[c1];
            if (mv2) e2 = H[c2];
            if (mv1) H[cur] = e1;
            if (mv2) H[c1] = e2;
            cur = mv2 ? c2 : (mv1 ? c1 : cur);
            const bool more = mv2;
#else
            const T a = H[l], b = H[l + 1];
            const int g = cur << 2;
            T q0, q1, q2, q3;
            if (g <= n) { q0 = H[g]; q1 = H[g + 1]; q2 = H[g + 2]; q3 = H[g + 3]; }
            const int k1 = (l + 1 <= n && !(a.key < b.key)) ? 1 : 0;
            const T e1 = k1 ? b : a;
            const bool mv1 = e1.key < last.key;
            const int c1 = l + k1;
            const int l2 = c1 << 1;
            const T a2 = k1 ? q2 : q0, b2 = k1 ? q3 : q1;
            const int k2 = (l2 + 1 <= n && !(a2.key < b2.key)) ? 1 : 0;
            const T e2 = k2 ? b2 : a2;
            const bool mv2 = mv1 && l2 <= n && e2.key < last.key;
            if (mv1) H[cur] = e1;
            if (mv2) H[c1] = e2;
            cur = mv2 ? l2 + k2 : (mv1 ? c1 : cur);
            const bool more = mv2;
#endif
            if (!more) break;
        }
        return cur;
    }
    __device__ WinEntry wpop() {
        const WinEntry top = WH()[1];
        WinEntry last = WH()[wsize];
        const int n = --wsize;
        const int cur = sift_down2(WH(), n, last);
        WH()[cur] = last;
        WF()[nfree++] = (uint16_t)(top.sb & 0xFFFF);
        ftop = (int)(top.sb & 0xFFFF);
        if constexpr (kCoop) __syncwarp();
        return top;
    }
    __device__ void ppush(double key, int vert, int level, int birth) {
        if (psize >= C.pcap) {
            flags |= kFlagQueueDrop;
            return;
        }
        if (psize >= C.pphys) {
            flags |= kFlagCapacity;
            return;
        }
        PsEntry e;
        e.key = key; e.vert = vert; e.lb = ((uint32_t)level << 8) | (uint32_t)(birth & 0xFF);
        if constexpr (kCoop) {
            sift_up(PH(), ++psize, e);
        } else {
            int cur = ++psize, p = cur >> 1;
            while (p > 0) {
                PsEntry pe = ph(p);
                if (!(pe.key > key)) break;
                ph(cur) = pe;
                cur = p;
                p = cur >> 1;
            }
            ph(cur) = e;
        }
        if (psize > st_maxp()) st_maxp() = psize;
    }
    __device__ PsEntry ppop() {
        const PsEntry top = PH()[1];
        PsEntry last = PH()[psize];
        const int n = --psize;
        const int cur = sift_down2(PH(), n, last);
        PH()[cur] = last;
        if constexpr (kCoop) __syncwarp();
        return top;
    }

    // -------------------------------------------------- source lifecycle
    __device__ void begin(int v, bool clear_all) {
        source = v;
        wsize = psize = nfree = nfresh = 0;
        ftop = 0;
        vcount = scount = 0;
        total = 0;
        flags = 0;
        st_windows() = st_pseudos() = st_generated() = st_maxw() = st_maxp() = 0;
        st_steps() = 0;
        src_birth = 0;
        done = false;
        pk_valid = false;
        if (clear_all) {
            clear_tables();  // every slot now carries epoch 0 = empty
            epoch = 1;
        } else {
            ++epoch;
            if (epoch == 0) ++epoch;
        }
        initialize();
    }
    __device__ void save_epoch(int gtid) { C.epochs[gtid] = epoch; }

    // write the birth of vertex slot s, keeping the source's cached birth
    __device__ __forceinline__ void set_birth(int s, int v, int b) {
        VT()[s].birth = b;
        if (v == source) src_birth = b;
    }

    // ICHDevice::Initialize, vertex source (ICHDevice.cu:525-581)
    __device__ void initialize() {
        const DevMesh& M = C.M;
        int start = __ldg(&M.vr[source].first);
        if (start < 0) {  // isolated vertex: the reference indexes edges[-1]
            flags |= kFlagUndefined;
            return;
        }
        int cur = start;
        int guard = 0;
        do {
            if (++guard > 1 << 20) { flags |= kFlagWatchdog; return; }
            HeRec hc = ld_he(M.he, cur);
            int op = nxt(cur);
            HeRec ho = ld_he(M.he, op);
            HeRec hp = ld_he(M.he, prv(cur));
            NewWin w;
            finish_window(0.0, ho.len, hc.len, hp.len, 0.0, w);
            w.p.cross = ho.twin;
            w.p.level = 0;
            wpush(w, source, 0);
            int opv = hc.v1;
            int s = vput(opv);
            if (s < 0) return;
            if (hc.len > VT()[s].dist) {
                cur = hc.twin;
                if (cur != -1) cur = nxt(cur);
                continue;
            }
            set_birth(s, opv, 0);
            VT()[s].dist = hc.len;
            VT()[s].enter = hc.twin;
            VT()[s].sslot = -1;
            if (!(__ldg(&M.vr[opv].flags) & kVertSaddleGE)) {
                cur = hc.twin;
                if (cur != -1) cur = nxt(cur);
                continue;
            }
            ppush(hc.len, opv, 0, VT()[s].birth);
            cur = hc.twin;
            if (cur != -1) cur = nxt(cur);
        } while (cur != start && cur != -1);
        int s = vput(source);
        if (s < 0) return;
        set_birth(s, source, 0);
        VT()[s].dist = 0.0;
        VT()[s].enter = -1;
        VT()[s].sslot = -1;
    }

    // ICHDevice::IsValidWindow (ICHDevice.cu:906-955) given the distances d1,
    // d2, d3 of the window half-edge's start, end and opposite vertex; l0 its
    // length; (tx,ty) the opposite vertex in the window's frame.
    __device__ __forceinline__ bool valid_window(const NewWin& w, bool isLeft, double d1, double d2, double d3,
                                                 double l0, double tx, double ty) const {
        const WinPay& p = w.p;
        if (p.b1 <= p.b0) return false;
        const double dB = hyp(p.sx - p.b1, p.sy - 0.0);
        const double dA = hyp(p.sx - p.b0, p.sy - 0.0);
        if (p.psd + dB > d1 + p.b1 && (p.psd + dB) / (d1 + p.b1) - 1.0 > 0.0) return false;
        if (p.psd + dA > d2 + l0 - p.b0 && (p.psd + dA) / (d2 + l0 - p.b0) - 1.0 > 0.0) return false;
        const double q = isLeft ? hyp(tx - p.b0, ty - 0.0) : hyp(tx - p.b1, ty - 0.0);
        const double dd = isLeft ? dA : dB;
        const double thr = isLeft ? 0.0 : kRelErr;
        if (p.psd + dd > d3 + q && (p.psd + dd) / (d3 + q) - 1.0 > thr) return false;
        return true;
    }

    // ICHDevice::BuildWindow (ICHDevice.cu:957-973); (v0x,v0y)-(v1x,v1y) is the
    // child's half-edge in the parent's frame, cross the twin of that half-edge.
    __device__ __forceinline__ void build_window(const WinPay& f, int cross, double elen, double t0, double t1,
                                                 double v0x, double v0y, double v1x, double v1y, NewWin& w) {
        double b0 = (1 - t0) * elen, b1 = (1 - t1) * elen;
        double px = v0x * t0 + v1x * (1 - t0), py = v0y * t0 + v1y * (1 - t0);
        double d0 = hyp(f.sx - px, f.sy - py);
        px = v0x * t1 + v1x * (1 - t1);
        py = v0y * t1 + v1y * (1 - t1);
        double d1 = hyp(f.sx - px, f.sy - py);
        finish_window(b0, b1, d0, d1, f.psd, w);
        w.p.cross = cross;
        w.p.level = f.level + 1;
    }

    // ICHDevice::PropagateWindow (ICHDevice.cu:618-726).  The face beyond the
    // window is e0 -> e1 -> e2 (e0 = twin of the window's half-edge) with
    // vertices A = v0(e0), B = v1(e0) and the opposite vertex C = v1(e1).  The
    // child on e1 (B->C) tests its validity against B, C, A and the child on
    // e2 (C->A) against C, A, B, so the three distances are probed once, in
    // parallel with the split entry of e0, and both children are built by one
    // code path: child 0 = left (frame (0,0)->apex), child 1 = right (frame
    // apex->(l0,0)).
    // All lanes of `amask` call this together and meet at each __syncwarp, so
    // the phases run converged; a lane with nothing to do (live == false, or a
    // boundary edge, or a full table) only predicates its work off.
    __device__ void propagate(const WinPay& win, int psrc, int birth, bool live, unsigned amask) {
        const DevMesh& M = C.M;
        const int e0 = win.cross;
        live = live && e0 != -1;
        int e1 = 0, e2 = 0, A = 0, B = 0, Cv = 0;
        HeRec h0, h1, h2;
        double2 v2 = make_double2(0.0, 0.0), top1 = v2, top2 = v2;
        uint32_t hA = 0, hB = 0, hC = 0, hS = 0;
        int4 kA = make_int4(0, 0, 0, 0), kB = kA, kC = kA, kS = kA;
        double dA = 0.0, dB = 0.0, dC = 0.0;
        double2 sdx = v2;
        int sC = -1, sS = -1;
        if (live) {
            e1 = nxt(e0);
            e2 = nxt(e1);
            h0 = ld_he(M.he, e0);
            h1 = ld_he(M.he, e1);
            h2 = ld_he(M.he, e2);
            v2 = ld_apex(M.geo, e0);
            top1 = ld_top(M.geo, e1);
            top2 = ld_top(M.geo, e2);
            A = h0.v0;
            B = h0.v1;
            Cv = h1.v1;
            if constexpr (!kCoop) {
                vfirst(A, hA, kA, dA);
                vfirst(B, hB, kB, dB);
                vfirst(Cv, hC, kC, dC);
                sfirst(e0, hS, kS, sdx);
                vfinish(A, hA, kA, dA);
                vfinish(B, hB, kB, dB);
                sC = vfinish(Cv, hC, kC, dC);
                sS = sfinish(e0, hS, kS, sdx);
            }
        }
        if constexpr (kCoop) {  // the four lookups in one group probe (live is the same in every thread)
            ProbeR ra, rb, rc, rs;
            coop_probe4(probe_q(VT(), C.vcap_log2, (uint32_t)A, live), probe_q(VT(), C.vcap_log2, (uint32_t)B, live),
                        probe_q(VT(), C.vcap_log2, (uint32_t)Cv, live), probe_q(ST(), C.scap_log2, (uint32_t)e0, live),
                        epoch, ra, rb, rc, rs);
            dA = ra.slot >= 0 ? __hiloint2double(ra.tail.y, ra.tail.x) : DBL_MAX;
            dB = rb.slot >= 0 ? __hiloint2double(rb.tail.y, rb.tail.x) : DBL_MAX;
            dC = rc.slot >= 0 ? __hiloint2double(rc.tail.y, rc.tail.x) : DBL_MAX;
            sC = rc.slot;
            kC = rc.head;
            sS = rs.slot;
            sdx = rs.slot >= 0 ? make_double2(__hiloint2double(rs.tail.y, rs.tail.x),
                                              __hiloint2double(rs.tail.w, rs.tail.z))
                               : make_double2(DBL_MAX, DBL_MAX);
        }
        __syncwarp(amask);

        const double sx = win.sx, sy = win.sy;
        const double l0 = h0.len;
        bool keep0 = live, keep1 = live, both = false;
        double interX = 0.0;
        if (live) {
            interX = v2.x - v2.y * (v2.x - sx) / (v2.y - sy);
            if (interX <= win.b0) {
                keep0 = false;  // right child only
            } else if (interX >= win.b1) {
                keep1 = false;  // left child only
            } else {
                both = true;
                const double D = hyp(v2.x - sx, v2.y - sy) + win.psd;
                const double sd = sdx.x;
                if (D > sd && D / sd - 1.0 > kRelErr) {  // one angle, one split
                    keep0 = sdx.y < interX;
                    keep1 = !keep0;
                } else {
                    int ssl = sS;
                    bool ok = true;
                    if (D < sd) {
#if SVG_INSERT_AT
                        // the lookup's chain ended at the empty slot (hS)
                        ssl = sS >= 0 ? sS : (kCoop ? sput(e0) : sinsert(e0, hS));
#else
                        ssl = sS >= 0 ? sS : sput(e0);
#endif
                        if (ssl < 0) {
                            ok = false;  // table full: the source goes to the retry pass
                        } else {
                            ST()[ssl].dist = D;
                            ST()[ssl].psrc = psrc;
                            ST()[ssl].x = l0 - interX;
                        }
                    }
                    if (ok && D < dC) {
                        if (dC == DBL_MAX) ++total;
#if SVG_INSERT_AT
                        const int s = sC >= 0 ? sC : (kCoop ? vput(Cv) : vinsert(Cv, hC));
#else
                        const int s = sC >= 0 ? sC : vput(Cv);
#endif
                        if (s < 0) {
                            ok = false;
                        } else {
                            const int b = (int)(signed char)((sC >= 0 ? kC.w : -1) + 1);
                            set_birth(s, Cv, b);
                            VT()[s].dist = D;
                            VT()[s].enter = e0;
                            VT()[s].sslot = ssl;  // D < dC <= split distance: the entry was just written
                            dC = D;  // the children's tests read the updated distance
                            if (__ldg(&M.vr[Cv].flags) & kVertSaddleGT) ppush(D, Cv, win.level + 1, b);
                        }
                    }
                    if (!ok) keep0 = keep1 = false;
                }
            }
        }
        __syncwarp(amask);

#if SVG_SEQ_CHILD
        // One child at a time through one copy of the code: build, test,
        // push.  The tests read only the three distances, which a push does
        // not change, so the heap sees the pushes in the same order.
#pragma unroll 1
        for (int c = 0; c < 2; ++c) {
            const bool left = c == 0;
            bool keep = left ? keep0 : keep1;
            NewWin W;
            if (keep) {
                // child 0: frame (0,0) -> apex; child 1: apex -> (l0,0)
                const double f0x = left ? 0.0 : v2.x, f0y = left ? 0.0 : v2.y;
                const double f1x = left ? v2.x : l0, f1y = left ? v2.y : 0.0;
                const bool fix0 = !left && both, fix1 = left && both;
                const double t0 = fix0 ? 1.0 : isect(sx, sy, win.b0, 0.0, f0x, f0y, f1x, f1y);
                const double t1 = fix1 ? 0.0 : isect(sx, sy, win.b1, 0.0, f0x, f0y, f1x, f1y);
                const double elen = left ? h1.len : h2.len;
                build_window(win, left ? h1.twin : h2.twin, elen, t0, t1, f0x, f0y, f1x, f1y, W);
                keep = left ? valid_window(W, true, dB, dC, dA, elen, top1.x, top1.y)
                            : valid_window(W, false, dC, dA, dB, elen, top2.x, top2.y);
            }
            __syncwarp(amask);
            if (keep) wpush(W, psrc, birth);
            __syncwarp(amask);
        }
    }
#else
        NewWin W0, W1;
        if (keep0) {
            const double t0 = isect(sx, sy, win.b0, 0.0, 0.0, 0.0, v2.x, v2.y);
            const double t1 = both ? 0.0 : isect(sx, sy, win.b1, 0.0, 0.0, 0.0, v2.x, v2.y);
            build_window(win, h1.twin, h1.len, t0, t1, 0.0, 0.0, v2.x, v2.y, W0);
            keep0 = valid_window(W0, true, dB, dC, dA, h1.len, top1.x, top1.y);
        }
        if (keep1) {
            const double t0 = both ? 1.0 : isect(sx, sy, win.b0, 0.0, v2.x, v2.y, l0, 0.0);
            const double t1 = isect(sx, sy, win.b1, 0.0, v2.x, v2.y, l0, 0.0);
            build_window(win, h2.twin, h2.len, t0, t1, v2.x, v2.y, l0, 0.0, W1);
            keep1 = valid_window(W1, false, dC, dA, dB, h2.len, top2.x, top2.y);
        }
        __syncwarp(amask);
        if (keep0) wpush(W0, psrc, birth);
        __syncwarp(amask);
        if (keep1) wpush(W1, psrc, birth);
        __syncwarp(amask);
    }
#endif

    // Fan walks of GenSubWinsForPseudoSrcFrom{Window,PseudoSrc}
    // (ICHDevice.cu:821-857, 867-903) with precomputed corner angles.
    __device__ void fan_walk(int left, int right, double a0, double a1, int& startEdge, int& endEdge) {
        const DevMesh& M = C.M;
        startEdge = -1;
        endEdge = -1;
        int cur = left;
        int guard = 0;
        while (a0 < kRefPi && cur != -1) {
            int nx = nxt(nxt(cur));
            a0 += ld_he(M.he, cur).corner;
            cur = ld_he(M.he, nx).twin;
            if (++guard > 1 << 20) { flags |= kFlagWatchdog; return; }
        }
        if (cur != -1) startEdge = nxt(ld_he(M.he, cur).twin);
        cur = right;
        while (a1 < kRefPi && cur != -1) {
            int nx = nxt(cur);
            a1 += ld_he(M.he, nx).corner;
            cur = ld_he(M.he, nx).twin;
            if (++guard > 1 << 20) { flags |= kFlagWatchdog; return; }
        }
        if (cur != -1) endEdge = ld_he(M.he, nxt(nxt(ld_he(M.he, cur).twin))).twin;
    }

    // ICHDevice::GenSubWinsForPseudoSrc (ICHDevice.cu:728-793).  Called by
    // the lanes of `amask` together (see propagate); `live` predicates.
    __device__ void gen_sub_wins(double pdist, int pv, int plevel, int pbirth, bool live, unsigned amask) {
        const DevMesh& M = C.M;
        int startEdge = -1, endEdge = -1;
        if (live) {
            int vs = vfind(pv);
            int enter = vs < 0 ? -1 : VT()[vs].enter;
            int vb = vs < 0 ? -1 : VT()[vs].birth;
            if (enter == -1 && vb != -1) {
                startEdge = __ldg(&M.vr[pv].first);
                endEdge = startEdge;
            } else if (enter >= 0 && ld_he(M.he, enter).v0 == pv) {
                fan_walk(enter, ld_he(M.he, enter).twin, 0.0, 0.0, startEdge, endEdge);
            } else if (enter >= 0 && ld_he(M.he, nxt(enter)).v1 == pv) {
                // GenSubWinsForPseudoSrcFromWindow (ICHDevice.cu:795-858)
                int e0 = enter, e1 = nxt(e0), e2 = nxt(e1);
                HeRec h0 = ld_he(M.he, e0), h1 = ld_he(M.he, e1), h2 = ld_he(M.he, e2);
                double l0 = h0.len, l1 = h1.len, l2 = h2.len;
                int ss = sfind(e0);
                double sx = ss < 0 ? DBL_MAX : ST()[ss].x;
                double ex = l0 - sx, ey = 0.0;
                double2 v2 = ld_apex(M.geo, e0);
                double dx = ex - v2.x, dy = ey - v2.y;
                double dl = hyp(dx, dy);
                double a0 = (dx * (0.0 - v2.x) + dy * (0.0 - v2.y)) / dl / l1;
                double a1 = (dx * (l0 - v2.x) + dy * (0.0 - v2.y)) / dl / l2;
                if (a0 > 1.0) a0 = 1.0; else if (a0 < -1.0) a0 = -1.0;
                if (a1 > 1.0) a1 = 1.0; else if (a1 < -1.0) a1 = -1.0;
                a0 = acos(a0);
                a1 = acos(a1);
                fan_walk(h1.twin, h2.twin, a0, a1, startEdge, endEdge);
            } else {
                flags |= kFlagUndefined;  // assert(false) at ICHDevice.cu:740
                live = false;
            }
            if (flags & kFlagWatchdog) live = false;
        }
        __syncwarp(amask);
        if (live) {
            int guard = 0;
            do {
                if (startEdge < 0) {  // the reference reads edges[-1] here
                    flags |= kFlagUndefined;
                    break;
                }
                int we = nxt(startEdge);
                HeRec hs = ld_he(M.he, startEdge), hw = ld_he(M.he, we);
                HeRec hn = ld_he(M.he, nxt(we));
                NewWin w;
                finish_window(0.0, hw.len, hs.len, hn.len, pdist, w);
                w.p.cross = hw.twin;
                w.p.level = plevel + 1;
                wpush(w, pv, pbirth);
                startEdge = hn.twin;
                if (++guard > 1 << 20) { flags |= kFlagWatchdog; live = false; break; }
            } while (startEdge != endEdge);
        }
        __syncwarp(amask);
        if (live) {
            int start = __ldg(&M.vr[pv].first), cur = start;
            int guard = 0;
            do {
                if (++guard > 1 << 20) { flags |= kFlagWatchdog; break; }
                HeRec hc = ld_he(M.he, cur);
                int opv = hc.v1;
                int os = vfind(opv);
                double od = os < 0 ? DBL_MAX : VT()[os].dist;
                if (!(__ldg(&M.vr[opv].flags) & kVertSaddleGE) || od < pdist + hc.len) {
                    cur = hc.twin;
                    if (cur != -1) cur = nxt(cur);
                    continue;
                }
                if (od == DBL_MAX) ++total;
                int s = os < 0 ? vput(opv) : os;
                if (s < 0) break;
                VT()[s].dist = pdist + hc.len;
                int b = (int)(signed char)(VT()[s].birth + 1);
                set_birth(s, opv, b);
                VT()[s].enter = hc.twin;
                VT()[s].sslot = -1;
                ppush(VT()[s].dist, opv, plevel, b);
                cur = hc.twin;
                if (cur != -1) cur = nxt(cur);
            } while (cur != start && cur != -1);
        }
        __syncwarp(amask);
    }

    // One iteration of ICHDevice::Execute's loop (ICHDevice.cu:72-119),
    // split into peek() - which entry comes off next - and act() - pop it
    // and process it.  The reference first pops every outdated window, then
    // every outdated pseudo-source (birth time no longer that of its
    // pseudo-source vertex, :80-86), then processes the smaller top; here one
    // outdated entry is popped per action, in the same order, which removes
    // the same entries (those pops change nothing else), and a processing
    // action follows once both tops are current.
    //   kActWindow  pop the window top (outdated, or processed: PropagateWindow)
    //   kActPseudo  pop the pseudo-source top (outdated, or GenSubWinsForPseudoSrc)
    //   kActDone    the source is finished
    // peek() caches its decision until act() runs, so a lane may wait.
    enum { kActWindow = 0, kActPseudo = 1, kActDone = 2 };
    bool done;
    bool pk_valid;
    int pk_act;
    bool pk_proc;  // process (true) or just drop an outdated entry (false)
#if SVG_SMEM_STATE
    __device__ __forceinline__ void set_pk(const WinEntry& w, const PsEntry& p) const {
        const int t = threadIdx.x;
        g_lane_smem.wkey[t] = w.key; g_lane_smem.wpsrc[t] = w.psrc; g_lane_smem.wsb[t] = w.sb;
        g_lane_smem.pkey[t] = p.key; g_lane_smem.pvert[t] = p.vert; g_lane_smem.plb[t] = p.lb;
    }
    __device__ __forceinline__ WinEntry pk_w() const {
        const int t = threadIdx.x;
        WinEntry w;
        w.key = g_lane_smem.wkey[t]; w.psrc = g_lane_smem.wpsrc[t]; w.sb = g_lane_smem.wsb[t];
        return w;
    }
    __device__ __forceinline__ PsEntry pk_p() const {
        const int t = threadIdx.x;
        PsEntry p;
        p.key = g_lane_smem.pkey[t]; p.vert = g_lane_smem.pvert[t]; p.lb = g_lane_smem.plb[t];
        return p;
    }
#else
    WinEntry pkw_;
    PsEntry pkp_;
    __device__ __forceinline__ void set_pk(const WinEntry& w, const PsEntry& p) { pkw_ = w; pkp_ = p; }
    __device__ __forceinline__ WinEntry pk_w() const { return pkw_; }
    __device__ __forceinline__ PsEntry pk_p() const { return pkp_; }
#endif

    // Up to this many outdated tops (pseudo-source reborn since the entry was
    // queued) are popped inside peek() instead of spending a voted step each;
    // the lane's heap operations happen in the same order either way.
    // The batched kernel passes SVG_ICH_INLINE_STALE; a lane stepping on its
    // own (the plain form) gains nothing from it and passes 0, which compiles
    // to a single look at the tops.
    template <int kInlineStale>
    __device__ int peek() {
        if (pk_valid) return pk_act;
        pk_valid = true;
        for (int inl = 0;; ++inl) {
            const int a = peek_once();
            if (a == kActDone || pk_proc || inl >= kInlineStale) return a;
            if (a == kActWindow) wpop();   // what act_window does with an outdated top
            else ppop();                   // likewise act_pseudo
        }
    }

    __device__ int peek_once() {
        pk_proc = false;
        if (done || (wsize == 0 && psize == 0) || (flags & (kFlagCapacity | kFlagWatchdog | kFlagUndefined))) {
            done = true;
            return pk_act = kActDone;
        }
        if (++st_steps() > C.watchdog) {
            flags |= kFlagWatchdog;
            done = true;
            return pk_act = kActDone;
        }
        WinEntry pw;
        PsEntry pp;
        pw.key = 0.0; pw.psrc = 0; pw.sb = 0;
        pp.key = 0.0; pp.vert = 0; pp.lb = 0;
        if (wsize > 0) pw = WH()[1];
        if (psize > 0) pp = PH()[1];
        set_pk(pw, pp);
        // both birth lookups issued together
        const bool wlook = wsize > 0 && pw.psrc != source;
        const bool plook = psize > 0;
        int wb = src_birth, pb = -1;
        if constexpr (kCoop) {
            ProbeR rw, rp, r2, r3;
            coop_probe4(probe_q(VT(), C.vcap_log2, (uint32_t)pw.psrc, wlook),
                        probe_q(VT(), C.vcap_log2, (uint32_t)pp.vert, plook), probe_off(), probe_off(), epoch, rw,
                        rp, r2, r3);
            if (wlook) wb = rw.slot < 0 ? -1 : rw.head.w;
            if (plook) pb = rp.slot < 0 ? -1 : rp.head.w;
        } else {
            uint32_t hw = 0, hp = 0;
            int4 kw = make_int4(0, 0, 0, 0), kp = make_int4(0, 0, 0, 0);
            double dw = 0.0, dp = 0.0;
            if (wlook) vfirst(pw.psrc, hw, kw, dw);
            if (plook) vfirst(pp.vert, hp, kp, dp);
            if (wlook) wb = vfinish(pw.psrc, hw, kw, dw) < 0 ? -1 : kw.w;
            if (plook) pb = vfinish(pp.vert, hp, kp, dp) < 0 ? -1 : kp.w;
        }
        const bool wstale = wsize > 0 && (int)(signed char)(pw.sb >> 16) != wb;
        if (wstale) return pk_act = kActWindow;
        const bool pstale = psize > 0 && (int)(signed char)(pp.lb & 0xFF) != pb;
        if (pstale) return pk_act = kActPseudo;
        pk_proc = true;
        if (wsize > 0 && (psize == 0 || pw.key < pp.key)) return pk_act = kActWindow;
        if (psize > 0 && (wsize == 0 || pw.key >= pp.key)) return pk_act = kActPseudo;
        flags |= kFlagWatchdog;  // NaN keys: neither branch is taken; the reference spins
        done = true;
        return pk_act = kActDone;
    }

    // Pop the window top; process it if peek() said so.  The lanes of amask
    // call this together (each of them with its own top).
    __device__ void act_window(unsigned amask) {
        pk_valid = false;
        const bool proc = pk_proc;
        const WinEntry t = pk_w();
        WinPay pay;
        pay.cross = -1;
        pay.level = 0;
        if (proc) pay = WP()[t.sb & 0xFFFF];  // issued before the sift-down
        wpop();
        __syncwarp(amask);
        const bool live = proc && !(pay.level > C.M.nf);
        if (live) ++st_windows();
        propagate(pay, t.psrc, (int)(signed char)(t.sb >> 16), live, amask);
        if (live && C.K != -1 && total >= C.K) done = true;
    }

    __device__ void act_pseudo(unsigned amask) {
        pk_valid = false;
        const bool proc = pk_proc;
        const PsEntry t = pk_p();
        ppop();
        __syncwarp(amask);
        const int level = (int)(t.lb >> 8);
        const bool live = proc && !(level >= C.M.nf);
        if (live) ++st_pseudos();
        gen_sub_wins(t.key, t.vert, level, (int)(signed char)(t.lb & 0xFF), live, amask);
        if (live && C.K != -1 && total >= C.K) done = true;
    }

    // peek + act for one lane on its own (or, cooperative, for the whole
    // warp on its source); true when finished.
    __device__ bool step() {
        const unsigned self = kCoop ? 0xFFFFFFFFu : 1u << (threadIdx.x & 31);
        const int a = peek<0>();
        if (a == kActDone) return true;
        if (a == kActWindow) act_window(self);
        else act_pseudo(self);
        return false;
    }
};
using Lane = LaneT<false>;
using CoopLane = LaneT<true>;

// ICHDevice::BuildGeodesicPathTo(vertex) (ICHDevice.cu:336-480) for a
// vertex whose path reaches the source through windows only: walk back from
// key point (ee, x) across faces until the source is the opposite vertex.
// Outputs the last key point (next to the source); -1 if there is none.
__device__ __forceinline__ void trace_direct(const DevMesh& M, int source, int ee, double x, uint32_t& src_edge,
                                             double& src_x, int& flags) {
    src_edge = 0xFFFFFFFFu;
    src_x = 0.0;
    int gid = ee;
    double gpos = x;
    HeRec hg = ld_he(M.he, gid);
    if (hg.twin < 0) { flags |= kFlagUndefined; return; }
    int opv = ld_he(M.he, nxt(hg.twin)).v1;
    double2 last = ld_apex(M.geo, gid);
    double cx = hg.len - gpos, cy = 0.0;
    int guard = 0;
    while (opv != source) {
        if (++guard > M.nf + 8) { flags |= kFlagWatchdog; return; }
        int e0 = hg.twin, e1 = nxt(e0), e2 = nxt(e1);
        double L0 = ld_he(M.he, e0).len, L1 = ld_he(M.he, e1).len, L2 = ld_he(M.he, e2).len;
        double2 ov = ld_top(M.geo, e0);
        double s = gpos / L0, t = 1.0 - gpos / L0;
        double2 nl;
        if (to_left(ov.x, ov.y, last.x, last.y, cx, cy)) {
            double2 p0 = ld_apex(M.geo, e1);
            nl.x = p0.x * s + L1 * t;
            nl.y = p0.y * s + 0.0 * t;
            gpos = isect(last.x, last.y, cx, cy, L0, 0.0, ov.x, ov.y);
            gpos = (1.0 - gpos) * L1;
            gid = e1;
            cx = L1 - gpos;
        } else {
            double2 p1 = ld_apex(M.geo, e2);
            nl.x = 0.0 * s + p1.x * t;
            nl.y = 0.0 * s + p1.y * t;
            gpos = isect(last.x, last.y, cx, cy, ov.x, ov.y, 0.0, 0.0);
            gpos = (1.0 - gpos) * L2;
            gid = e2;
            cx = L2 - gpos;
        }
        cy = 0.0;
        last = nl;
        src_edge = (uint32_t)gid;
        src_x = gpos;
        hg = ld_he(M.he, gid);
        if (hg.twin < 0) { flags |= kFlagUndefined; return; }
        opv = ld_he(M.he, nxt(hg.twin)).v1;
    }
}

}  // namespace svgb
