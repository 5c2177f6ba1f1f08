// Test-oracle driver around the REFERENCE's own ICH engine, compiled as host
// C++ from the reference sources where they lie (Mesh.cu, Geometry.cu,
// ICHDevice.cu; see oracle/Makefile).  This file is test infrastructure: only
// tests/, the smoke check and bench.py's CPU-baseline leg load the library it
// builds (oracle/_ref/libsvgref.so).  It is never part of the product.
//
// What is restated here (the only reference code that cannot be compiled
// with g++ because it sits in a __global__ kernel / <<<>>> launch file):
//   * the per-source body of constructSVG       SVG.cu:34-76
//   * the per-thread buffer set-up              SVG.cu:18-29, SVG.cu:119-140
//   * SolveSSSD / SolveMSAD / Astar (host path) SVG.cu:241-251, 354-413
// Everything else (mesh loading, ICH window propagation, queues, hash tables,
// geodesic back-trace) is the reference's compiled code, called unchanged.
//
// Boundary handling: Mesh::LoadFromFile (Mesh.cu:62-90) never marks boundary
// half-edges; vector::resize leaves their twinEdge at 0.  ref_mesh_load with
// fix_boundary=1 re-derives which half-edges were paired by the same
// (min,max)-vertex rule and sets the others to -1, i.e. the one-line
// "twinEdge = -1 at Mesh.cu:76" variant.  On closed meshes it changes nothing.

#include "Mesh.cuh"
#include "ICHDevice.cuh"
#include "PriorityQueueWithHandle.cuh"

#include <atomic>
#include <chrono>
#include <cstdint>
#include <map>
#include <thread>
#include <vector>

namespace {

// Same byte layout as SVG::SVGNode (SVG.cuh:21-27): 40 bytes on x86-64.
struct RefNode {
    int adjNode;
    double geodDist;
    unsigned nextToSrcEdge, nextToDstEdge;
    double nextToSrcX, nextToDstX;
};
static_assert(sizeof(RefNode) == 40, "SVGNode layout");

// Reference constants (SVG.cuh:13-16).
constexpr int kWinPQSize = 1024;
constexpr int kPseudoPQSize = 1024;
constexpr int kStoredWinBuf = 100;
constexpr int kKeptFaces = 10;

struct IchScratch {
    std::vector<PriorityQueues<ICHDevice::Window>::PQItem> win;
    std::vector<PriorityQueues<ICHDevice::PseudoWindow>::PQItem> pseudo;
    std::vector<ICHDevice::SplitItem> split;
    std::vector<ICHDevice::VertItem> vert;
    std::vector<ICHDevice::Window> stored;
    std::vector<unsigned> kept;
    ICHDevice ich;

    // Mirrors the per-thread slice set-up of constructSVG (SVG.cu:18-29).
    IchScratch(Mesh* mesh, unsigned splitSize, unsigned vertSize, int winCap, int pseudoCap)
        : win(winCap + 1), pseudo(pseudoCap + 1), split(splitSize + 1), vert(vertSize + 1),
          stored(kStoredWinBuf), kept(kKeptFaces) {
        PriorityQueues<ICHDevice::Window> winPQ(winCap);
        PriorityQueues<ICHDevice::PseudoWindow> pseudoPQ(pseudoCap);
        winPQ.AssignMemory(win.data(), winCap);
        pseudoPQ.AssignMemory(pseudo.data(), pseudoCap);
        ich.AssignMesh(mesh);
        ich.AssignBuffers(split.data(), splitSize, vert.data(), vertSize, winPQ, pseudoPQ,
                          stored.data(), kept.data());
    }
};

int clamp_threads(int n) {
    if (n <= 0) n = (int)std::thread::hardware_concurrency();
    return n < 1 ? 1 : n;
}

}  // namespace

extern "C" {

void* ref_mesh_load(const char* path, int fix_boundary) {
    Mesh* m = new Mesh();
    if (!m->LoadFromFile(path)) {
        delete m;
        return nullptr;
    }
    if (fix_boundary) {
        std::vector<char> paired(m->edgeNum, 0);
        std::map<std::pair<int, int>, int> first;
        for (int e = 0; e < m->edgeNum; ++e) {
            int a = m->edges[e].verts[0], b = m->edges[e].verts[1];
            if (a > b) std::swap(a, b);
            auto it = first.find({a, b});
            if (it != first.end()) {
                paired[e] = 1;
                paired[it->second] = 1;
            } else {
                first[{a, b}] = e;
            }
        }
        for (int e = 0; e < m->edgeNum; ++e)
            if (!paired[e]) m->edges[e].twinEdge = -1;
    }
    return m;
}

void ref_mesh_free(void* h) {
    Mesh* m = static_cast<Mesh*>(h);
    if (!m) return;
    m->clear();
    delete m;
}

void ref_mesh_counts(void* h, int* nv, int* nf, int* ne) {
    Mesh* m = static_cast<Mesh*>(h);
    *nv = m->vertNum;
    *nf = m->faceNum;
    *ne = m->edgeNum;
}

// Export the loaded half-edge structure (for checking the product's loader).
void ref_mesh_export(void* h, double* pos, int* faces, int* he_v0, int* he_v1, int* he_twin,
                     int* he_next, int* he_prev, int* he_face, double* he_len, double* angle,
                     int* first_edge) {
    Mesh* m = static_cast<Mesh*>(h);
    for (int v = 0; v < m->vertNum; ++v) {
        if (pos) {
            pos[3 * v] = m->verts[v].pos.x;
            pos[3 * v + 1] = m->verts[v].pos.y;
            pos[3 * v + 2] = m->verts[v].pos.z;
        }
        if (angle) angle[v] = m->verts[v].angle;
        if (first_edge) first_edge[v] = m->verts[v].firstEdge;
    }
    for (int f = 0; f < m->faceNum && faces; ++f)
        for (int j = 0; j < 3; ++j) faces[3 * f + j] = (int)m->faces[f].verts[j];
    for (int e = 0; e < m->edgeNum; ++e) {
        if (he_v0) he_v0[e] = m->edges[e].verts[0];
        if (he_v1) he_v1[e] = m->edges[e].verts[1];
        if (he_twin) he_twin[e] = m->edges[e].twinEdge;
        if (he_next) he_next[e] = m->edges[e].nextEdge;
        if (he_prev) he_prev[e] = m->edges[e].prevEdge;
        if (he_face) he_face[e] = m->edges[e].faceId;
        if (he_len) he_len[e] = m->edges[e].edgeLen;
    }
}

// Build the SVG rows of `nsrc` sources with the reference's ICH.
//   nodes  : nsrc*K RefNode slots (row r holds tails[r] entries), padded like d_svg.
//   stats  : nsrc*4 ints {numOfWinGen, maxWinQSize, maxPseudoQSize, totalCalcVertNum}, or NULL.
//   win_cap/pseudo_cap: queue capacities; the reference uses 1023 (SVG.cu:18-21).
// Returns wall seconds spent in the source loop (all threads).
double ref_build(void* h, int K, unsigned splitCoef, unsigned vertCoef, int win_cap, int pseudo_cap,
                 const int* sources, int nsrc, int nthreads, int* tails, void* nodes_out, int* stats) {
    Mesh* mesh = static_cast<Mesh*>(h);
    RefNode* nodes = static_cast<RefNode*>(nodes_out);
    nthreads = clamp_threads(nthreads);
    if (nthreads > nsrc) nthreads = nsrc > 0 ? nsrc : 1;
    std::atomic<int> next(0);
    auto t0 = std::chrono::steady_clock::now();
    auto worker = [&]() {
        IchScratch s(mesh, (unsigned)K * splitCoef, (unsigned)K * vertCoef, win_cap, pseudo_cap);
        ICHDevice& ich = s.ich;
        for (;;) {
            int r = next.fetch_add(1);
            if (r >= nsrc) break;
            int i = sources[r];
            // ---- SVG.cu:36-75, restated ----
            ich.Clear();
            ich.AddSource(i);
            ich.Execute(K);
            int tail = 0;
            RefNode* row = nodes + (size_t)K * r;
            for (int j = 0; j < mesh->vertNum; ++j) {
                if (ich.GetDistanceTo(j) == DBL_MAX) continue;
                if (j == i) continue;
                unsigned srcId;
                unsigned nextToSrcEdge, nextToDstEdge;
                // The reference leaves these uninitialised when the path has no
                // interior key point; fix them to 0.0 so outputs are deterministic.
                double nextSrcX = 0.0, nextDstX = 0.0;
                ich.BuildGeodesicPathTo(j, srcId, nextToSrcEdge, nextSrcX, nextToDstEdge, nextDstX);
                if (ich.pathPassVert) continue;
                if (nextToSrcEdge == (unsigned)-1) {
                    nextToSrcEdge = nextToDstEdge;
                    nextSrcX = nextDstX;
                }
                row[tail].adjNode = j;
                row[tail].geodDist = ich.GetDistanceTo(j);
                row[tail].nextToSrcX = nextSrcX;
                row[tail].nextToSrcEdge = nextToSrcEdge;
                row[tail].nextToDstX = nextDstX;
                row[tail].nextToDstEdge = nextToDstEdge;
                ++tail;
                if (tail == K) break;
            }
            tails[r] = tail;
            if (stats) {
                stats[4 * r + 0] = ich.numOfWinGen;
                stats[4 * r + 1] = ich.maxWinQSize;
                stats[4 * r + 2] = ich.maxPseudoQSize;
                stats[4 * r + 3] = ich.totalCalcVertNum;
            }
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nthreads; ++t) pool.emplace_back(worker);
    worker();
    for (auto& t : pool) t.join();
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// Per-vertex distances of the reference ICH from `nsrc` sources, K-limited
// (K > 0) or exhaustive (K = -1, the exact-ICH oracle), with caller-chosen
// table sizes and queue capacities.  dist_out is nsrc*V, DBL_MAX = unreached.
double ref_ich_distances(void* h, int K, unsigned splitSize, unsigned vertSize, int win_cap,
                         int pseudo_cap, const int* sources, int nsrc, int nthreads,
                         double* dist_out, int* stats) {
    Mesh* mesh = static_cast<Mesh*>(h);
    nthreads = clamp_threads(nthreads);
    if (nthreads > nsrc) nthreads = nsrc > 0 ? nsrc : 1;
    std::atomic<int> next(0);
    auto t0 = std::chrono::steady_clock::now();
    auto worker = [&]() {
        IchScratch s(mesh, splitSize, vertSize, win_cap, pseudo_cap);
        ICHDevice& ich = s.ich;
        for (;;) {
            int r = next.fetch_add(1);
            if (r >= nsrc) break;
            ich.Clear();
            ich.AddSource(sources[r]);
            ich.Execute(K);
            double* d = dist_out + (size_t)mesh->vertNum * r;
            for (int j = 0; j < mesh->vertNum; ++j) d[j] = ich.GetDistanceTo(j);
            if (stats) {
                stats[4 * r + 0] = ich.numOfWinGen;
                stats[4 * r + 1] = ich.maxWinQSize;
                stats[4 * r + 2] = ich.maxPseudoQSize;
                stats[4 * r + 3] = ich.totalCalcVertNum;
            }
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nthreads; ++t) pool.emplace_back(worker);
    worker();
    for (auto& t : pool) t.join();
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // extern "C"

// ---- Graph search, restated from SVG.cu:241-251 (SolveSSSD), 354-366
// (SolveMSAD) and 369-413 (Astar), on the padded V*K node array + tails. ----
struct SVG_GraphDist {  // SVG::GraphDistInfo (SVG.cuh:29-37)
    double dist;
    int pathParentIndex;
    int srcId;
    int indexInPQ;
};

extern "C" {
static void ref_astar(const Mesh* mesh, int K, const int* tails, const RefNode* svg, int t,
                      bool astar, SVG_GraphDist* g, PriorityQueuesWithHandle<int>& pq) {
    while (!pq.empty()) {
        int cur = pq.pop();
        if (astar && cur == t) {
            pq.clear();
            break;
        }
        const RefNode* row = svg + (size_t)K * cur;
        for (int i = 0; i < tails[cur]; ++i) {
            int adj = row[i].adjNode;
            double nd = g[cur].dist + row[i].geodDist;
            if (nd >= g[adj].dist) continue;
            g[adj].dist = nd;
            g[adj].pathParentIndex = cur;
            g[adj].srcId = g[cur].srcId;
            double pri = astar ? nd + (mesh->verts[adj].pos - mesh->verts[t].pos).length() : nd;
            if (g[adj].indexInPQ == -1)
                pq.push(adj, &g[adj].indexInPQ, pri);
            else
                pq.decrease(g[adj].indexInPQ, pri);
        }
    }
}

// SSSD A* for n (s,t) pairs.  dist_out[n]; parent_out (n*V, optional).
double ref_sssd(void* h, int K, const int* tails, const void* svg_nodes, int n, const int* s,
                const int* t, double* dist_out, int* hops_out) {
    Mesh* mesh = static_cast<Mesh*>(h);
    const RefNode* svg = static_cast<const RefNode*>(svg_nodes);
    int V = mesh->vertNum;
    std::vector<SVG_GraphDist> g(V);
    std::vector<PriorityQueuesWithHandle<int>::PQItem> buf(V + 1);
    PriorityQueuesWithHandle<int> pq(V);
    pq.AssignMemory(buf.data(), V);
    auto t0 = std::chrono::steady_clock::now();
    for (int q = 0; q < n; ++q) {
        for (int i = 0; i < V; ++i) g[i] = {DBL_MAX, -1, -1, -1};
        pq.clear();
        int ss = s[q], tt = t[q];
        g[ss].dist = 0.0;
        g[ss].pathParentIndex = -1;
        g[ss].srcId = ss;
        pq.push(ss, &g[ss].indexInPQ, 0.0 + (mesh->verts[ss].pos - mesh->verts[tt].pos).length());
        ref_astar(mesh, K, tails, svg, tt, true, g.data(), pq);
        dist_out[q] = g[tt].dist;
        if (hops_out) {
            int c = 0, v = tt;
            while (v != -1 && v != ss && c <= V) { v = g[v].pathParentIndex; ++c; }
            hops_out[q] = c;
        }
    }
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// MSAD Dijkstra for one weighted source set: dist_out[V], src_out[V] (optional).
double ref_msad(void* h, int K, const int* tails, const void* svg_nodes, int ns, const int* srcs,
                const double* weights, double* dist_out, int* src_out) {
    Mesh* mesh = static_cast<Mesh*>(h);
    const RefNode* svg = static_cast<const RefNode*>(svg_nodes);
    int V = mesh->vertNum;
    std::vector<SVG_GraphDist> g(V, {DBL_MAX, -1, -1, -1});
    std::vector<PriorityQueuesWithHandle<int>::PQItem> buf(V + 1);
    PriorityQueuesWithHandle<int> pq(V);
    pq.AssignMemory(buf.data(), V);
    auto t0 = std::chrono::steady_clock::now();
    for (int i = 0; i < ns; ++i) {
        g[srcs[i]].dist = weights[i];
        g[srcs[i]].pathParentIndex = -1;
        g[srcs[i]].srcId = srcs[i];
        pq.push(srcs[i], &g[srcs[i]].indexInPQ, weights[i]);
    }
    ref_astar(mesh, K, tails, svg, -1, false, g.data(), pq);
    for (int v = 0; v < V; ++v) {
        dist_out[v] = g[v].dist;
        if (src_out) src_out[v] = g[v].srcId;
    }
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // extern "C"
