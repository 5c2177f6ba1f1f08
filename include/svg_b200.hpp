/* svg_b200.hpp: the reference's Mesh / SVG host classes (Mesh.cuh:33-52,
 * SVG.cuh:18-113) as a header-only C++ wrapper over the C ABI of
 * svg_b200.h, so that a driver written against the reference (its
 * kernel.cu mains) compiles against this header with the same class names,
 * method names and argument order:
 *
 *     Mesh mesh, d_mesh;
 *     mesh.LoadFromFile(argv[1]);            // Mesh::LoadFromFile   (Mesh.cu:24)
 *     mesh.copyToGPU(&d_mesh);               // Mesh::copyToGPU      (Mesh.cu:128)
 *     SVG svg;
 *     svg.AssignMesh(&mesh, &d_mesh);        // SVG::AssignMesh      (SVG.cu:109)
 *     svg.SetParameters(K, 10, 2);           // SVG::SetParameters   (SVG.cu:114)
 *     svg.Allocation();                      // SVG::Allocation      (SVG.cu:119)
 *     svg.ConstructSVG();                    // SVG::ConstructSVG    (SVG.cu:160)
 *     svg.Free();                            // SVG::Free            (SVG.cu:142)
 *     svg.CopySVGToHost();                   // SVG::CopySVGToHost   (SVG.cu:184)
 *     svg.SaveSVGToFile("mesh.svg");         // SVG::SaveSVGToFile   (SVG.cu:208)
 *     svg.SolveSSSD(s, t, mesh, infos, pq);  // SVG::SolveSSSD       (SVG.cu:241)
 *     svg.SolveMSAD(src, w, n, mesh, infos, pq);  // SVG::SolveMSAD  (SVG.cu:354)
 *     svg.FreeSVGStructure(); mesh.clear(); d_mesh.clearGPU();
 *
 * Differences a caller can see:
 *  - Errors throw svg_b200::Error (what() = svg_last_error()) where the
 *    reference prints and exits (HANDLE_ERROR, book.cuh:23-33);
 *    LoadFromFile still returns false for a file it cannot open.
 *  - Like the reference's classes, Mesh and SVG are shallow handles with no
 *    destructor that frees: copies share the device objects, and clear() /
 *    clearGPU() / FreeSVGStructure() release them.  Mesh keeps one library
 *    mesh for the host and device sides; it is freed once both the host
 *    object and its device copy have been cleared (or the host object, if it
 *    was never copied).
 *  - The searches run on the GPU (batched kernels), so the caller's
 *    PriorityQueuesWithHandle is accepted and unused, and GraphDistInfo need
 *    not be reset between queries.  SolveSSSD fills dist, pathParentIndex and
 *    srcId of the vertices on the s-t path (t's entry holds the distance,
 *    as the reference's does); SolveMSAD fills every vertex.  Among equally
 *    short predecessors the smallest vertex id is named.
 *  - The host graph after CopySVGToHost is CSR (rows of at most K nodes,
 *    ascending neighbour id, exactly the reference's rows) instead of a V x K
 *    padded array; Degree(v) / Row(v) read it.
 *  - Extensions with no counterpart: SolveSSSDBatch / SolveMSADBatch (many
 *    queries per launch), Stats(), and Options() for the other build options.
 *
 * Link with -lsvg_b200 (the library links the CUDA runtime statically).
 * Define SVG_B200_NO_GLOBAL_NAMES to keep the classes inside namespace
 * svg_b200 instead of also naming them Mesh, SVG, Edge, Vertex, Face and
 * PriorityQueuesWithHandle at global scope.
 */
#ifndef SVG_B200_HPP
#define SVG_B200_HPP

#include <cfloat>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "svg_b200.h"

namespace svg_b200 {

struct Error : std::runtime_error {
    svg_status code;
    Error(svg_status c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void check(svg_status s) {
    if (s != SVG_OK) throw Error(s, svg_last_error());
}

/* Vector3D's fields (Geometry.cuh) as far as a driver reads positions. */
struct Vector3D {
    double x = 0.0, y = 0.0, z = 0.0;
};

/* Edge / Vertex / Face of Mesh.cuh:6-31 (half-edge 3f+j of face f). */
struct Edge {
    int verts[2];
    int twinEdge, nextEdge, prevEdge;
    int faceId;
    double edgeLen;
};
struct Vertex {
    Vector3D pos;
    double angle = 0.0;
    int firstEdge = -1;
};
struct Face {
    unsigned verts[3];
    unsigned edges[3];
};

class Mesh {
    struct Shared {
        svg_mesh* h = nullptr;
        bool host_cleared = false, device_made = false, device_cleared = false;
        std::vector<Edge> e;
        std::vector<Vertex> v;
        std::vector<Face> f;
        ~Shared() { /* released by clear() / clearGPU(), as the reference releases by hand */ }
        void release_if_done() {
            if (h && host_cleared && (!device_made || device_cleared)) {
                svg_mesh_free(h);
                h = nullptr;
            }
        }
    };
    std::shared_ptr<Shared> s_;
    bool device_side_ = false;

    void bind_arrays() {
        edges = s_->e.empty() ? nullptr : s_->e.data();
        verts = s_->v.empty() ? nullptr : s_->v.data();
        faces = s_->f.empty() ? nullptr : s_->f.data();
    }

public:
    Edge* edges = nullptr;
    int edgeNum = 0;
    Vertex* verts = nullptr;
    int vertNum = 0;
    Face* faces = nullptr;
    int faceNum = 0;

    /* Mesh::LoadFromFile (Mesh.cu:24-126): false if the file cannot be
     * opened; throws for a file that opens but is not a usable mesh. */
    bool LoadFromFile(const char* fileName) {
        svg_mesh* h = nullptr;
        svg_status st = svg_mesh_load_obj(fileName, &h);
        if (st == SVG_ERR_IO) return false;
        check(st);
        adopt(h);
        return true;
    }

    /* The same mesh from arrays (pos[3*nv], faces[3*nf], 0-based); no
     * counterpart in the reference, which only loads files. */
    void FromArrays(int32_t nv, const double* pos, int32_t nf, const int32_t* fv) {
        svg_mesh* h = nullptr;
        check(svg_mesh_from_arrays(nv, pos, nf, fv, &h));
        adopt(h);
    }

    /* Mesh::copyToGPU (Mesh.cu:128-142): d_mesh is a host object that stands
     * for the device copy, as in the reference. */
    bool copyToGPU(Mesh* d_mesh) {
        if (!s_ || !s_->h) throw Error(SVG_ERR_STATE, "copyToGPU: no mesh loaded");
        check(svg_mesh_upload(s_->h));
        s_->device_made = true;
        s_->device_cleared = false;
        if (d_mesh && d_mesh != this) {
            d_mesh->s_ = s_;
            d_mesh->device_side_ = true;
            d_mesh->vertNum = vertNum;
            d_mesh->faceNum = faceNum;
            d_mesh->edgeNum = edgeNum;
            d_mesh->bind_arrays();
        }
        return true;
    }

    /* Mesh::clear (Mesh.cu:144-150). */
    void clear() {
        if (s_ && !device_side_) {
            s_->host_cleared = true;
            s_->release_if_done();
        }
        drop();
    }

    /* Mesh::clearGPU (Mesh.cu:152-158), called on the device-side object. */
    void clearGPU() {
        if (s_ && device_side_) {
            s_->device_cleared = true;
            s_->release_if_done();
        }
        drop();
    }

    svg_mesh* handle() const { return s_ ? s_->h : nullptr; }

private:
    void adopt(svg_mesh* h) {
        int32_t nv = 0, nf = 0, ne = 0;
        check(svg_mesh_counts(h, &nv, &nf, &ne));
        auto sh = std::make_shared<Shared>();
        sh->h = h;
        std::vector<int32_t> v0((size_t)ne), twin((size_t)ne), first((size_t)nv);
        std::vector<double> len((size_t)ne), pos((size_t)nv * 3), ang((size_t)nv);
        check(svg_mesh_export(h, v0.data(), twin.data(), len.data(), pos.data(), ang.data(), first.data()));
        sh->e.resize((size_t)ne);
        for (int32_t e = 0; e < ne; ++e) {
            const int32_t f = e / 3, j = e % 3;
            const int32_t nx = 3 * f + (j + 1) % 3, pv = 3 * f + (j + 2) % 3;
            Edge& E = sh->e[(size_t)e];
            E.verts[0] = v0[(size_t)e];
            E.verts[1] = v0[(size_t)nx];
            E.twinEdge = twin[(size_t)e];
            E.nextEdge = nx;
            E.prevEdge = pv;
            E.faceId = f;
            E.edgeLen = len[(size_t)e];
        }
        sh->v.resize((size_t)nv);
        for (int32_t i = 0; i < nv; ++i) {
            Vertex& V = sh->v[(size_t)i];
            V.pos.x = pos[3 * (size_t)i];
            V.pos.y = pos[3 * (size_t)i + 1];
            V.pos.z = pos[3 * (size_t)i + 2];
            V.angle = ang[(size_t)i];
            V.firstEdge = first[(size_t)i];
        }
        sh->f.resize((size_t)nf);
        for (int32_t f = 0; f < nf; ++f)
            for (int j = 0; j < 3; ++j) {
                sh->f[(size_t)f].verts[j] = (unsigned)v0[(size_t)(3 * f + j)];
                sh->f[(size_t)f].edges[j] = (unsigned)(3 * f + j);
            }
        if (s_) clear();
        s_ = sh;
        device_side_ = false;
        vertNum = nv;
        faceNum = nf;
        edgeNum = ne;
        bind_arrays();
    }
    void drop() {
        s_.reset();
        edges = nullptr;
        verts = nullptr;
        faces = nullptr;
        vertNum = faceNum = edgeNum = 0;
    }
};

/* PriorityQueuesWithHandle (PriorityQueueWithHandle.cuh): the reference's
 * host searches need the caller's addressable heap; the GPU searches here
 * do not, so this keeps only the interface a driver calls. */
template <class T>
class PriorityQueuesWithHandle {
public:
    struct PQItem {
        double key;
        T item;
        int* backHandle;
    };
    PriorityQueuesWithHandle() {}
    explicit PriorityQueuesWithHandle(int /*maxSize*/) {}
    void AssignMemory(PQItem* /*buf*/, int /*maxSize*/) {}
    void clear() {}
};

class SVG {
public:
    /* SVG::SVGNode (SVG.cuh:21-27), the 40-byte record of svg_node. */
    struct SVGNode {
        int adjNode;
        double geodDist;
        unsigned nextToSrcEdge, nextToDstEdge;
        double nextToSrcX, nextToDstX;
    };
    /* SVG::GraphDistInfo (SVG.cuh:29-37). */
    struct GraphDistInfo {
        double dist;
        int pathParentIndex;
        int srcId;
        int indexInPQ;
        GraphDistInfo() : dist(DBL_MAX), pathParentIndex(-1), srcId(-1), indexInPQ(-1) {}
    };
    enum SEARCHTYPE { ASTAR, DIJKSTRA };

    SVG() { svg_build_opts_default(&opts_); }

    /* SVG::AssignMesh (SVG.cu:109-112). */
    void AssignMesh(Mesh* mesh_, Mesh* d_mesh_) {
        mesh = mesh_;
        d_mesh = d_mesh_;
    }
    /* SVG::SetParameters (SVG.cu:114-117). */
    void SetParameters(int K_, unsigned splitInfoCoef_, unsigned vertInfoCoef_) {
        K = K_;
        splitInfoCoef = splitInfoCoef_;
        vertInfoCoef = vertInfoCoef_;
    }
    /* SVG::Allocation (SVG.cu:119-140): the build sizes and holds its own
     * scratch (under svg_build_opts.hbm_budget), so nothing happens here. */
    bool Allocation() { return true; }
    /* SVG::Free (SVG.cu:142-147): scratch is released by the build. */
    void Free() {}
    /* SVG::FreeSVGStructure (SVG.cu:149-155). */
    void FreeSVGStructure() {
        if (g_) svg_graph_free(g_);
        g_ = nullptr;
        off_.clear();
        nodes_.clear();
    }

    /* SVG::ConstructSVG (SVG.cu:160-182): the batched build on the GPU. */
    void ConstructSVG() {
        svg_mesh* h = mesh_handle();
        FreeSVGStructure();
        opts_.K = K;
        opts_.split_coef = splitInfoCoef;
        opts_.vert_coef = vertInfoCoef;
        check(svg_build(h, &opts_, &g_));
    }

    /* SVG::CopySVGToHost (SVG.cu:184-206). */
    void CopySVGToHost() {
        need_graph();
        int32_t nv = 0, k = 0;
        int64_t nnz = 0;
        check(svg_graph_counts(g_, &nv, &nnz, &k));
        std::vector<int32_t> tails((size_t)nv);
        nodes_.assign((size_t)std::max<int64_t>(nnz, 1), SVGNode{});
        static_assert(sizeof(SVGNode) == sizeof(svg_node), "SVGNode is svg_node's 40-byte layout");
        check(svg_graph_copy_nodes(g_, tails.data(), reinterpret_cast<svg_node*>(nodes_.data())));
        nodes_.resize((size_t)nnz);
        off_.assign((size_t)nv + 1, 0);
        for (int32_t v = 0; v < nv; ++v) off_[(size_t)v + 1] = off_[(size_t)v] + tails[(size_t)v];
    }
    /* Row v of the host copy: Degree(v) nodes from Row(v). */
    int Degree(int v) const { return (int)(off_.at((size_t)v + 1) - off_.at((size_t)v)); }
    const SVGNode* Row(int v) const { return nodes_.data() + off_.at((size_t)v); }

    /* SVG::SaveSVGToFile / LoadSVGFromFile (SVG.cu:208-239): the reference's format. */
    void SaveSVGToFile(const char* fileName) {
        need_graph();
        check(svg_graph_save(g_, fileName));
    }
    void LoadSVGFromFile(const char* fileName) {
        svg_mesh* h = mesh_handle();
        FreeSVGStructure();
        check(svg_graph_load(h, K, fileName, &g_));
    }

    /* SVG::SolveSSSD(s, t, ...) (SVG.cu:241-251): the s-t distance in
     * graphDistInfos[t].dist and the path along pathParentIndex. */
    void SolveSSSD(int s, int t, Mesh /*mesh*/, GraphDistInfo* graphDistInfos, PriorityQueuesWithHandle<int> /*pq*/) {
        need_graph();
        searchType = ASTAR;
        std::vector<int32_t> path(1024);
        std::vector<double> pd(1024);
        int32_t len = 0;
        double d = DBL_MAX;
        svg_status st = svg_sssd_path(g_, s, t, (int32_t)path.size(), path.data(), pd.data(), &len, &d);
        if (st == SVG_ERR_ARG && len > (int32_t)path.size()) {
            path.resize((size_t)len);
            pd.resize((size_t)len);
            st = svg_sssd_path(g_, s, t, len, path.data(), pd.data(), &len, &d);
        }
        check(st);
        graphDistInfos[t].dist = d;
        for (int32_t i = 0; i < len; ++i) {
            GraphDistInfo& gi = graphDistInfos[path[(size_t)i]];
            gi.dist = pd[(size_t)i];
            gi.pathParentIndex = i + 1 < len ? path[(size_t)i + 1] : -1;
            gi.srcId = s;
        }
    }

    /* SVG::SolveMSAD (SVG.cu:354-366): every vertex's distance, source and
     * parent in graphDistInfos[0 .. vertNum). */
    void SolveMSAD(int* sources, double* sourceWeights, int Ns, Mesh /*mesh*/, GraphDistInfo* graphDistInfos,
                   PriorityQueuesWithHandle<int> /*pq*/) {
        need_graph();
        searchType = DIJKSTRA;
        int32_t nv = 0, k = 0;
        int64_t nnz = 0;
        check(svg_graph_counts(g_, &nv, &nnz, &k));
        const int64_t off[2] = {0, Ns};
        std::vector<double> d((size_t)nv);
        std::vector<int32_t> src((size_t)nv), par((size_t)nv);
        check(svg_msad_batch_paths(g_, 1, off, sources, sourceWeights, d.data(), src.data(), par.data()));
        for (int32_t v = 0; v < nv; ++v) {
            graphDistInfos[v].dist = d[(size_t)v];
            graphDistInfos[v].srcId = src[(size_t)v];
            graphDistInfos[v].pathParentIndex = par[(size_t)v];
            graphDistInfos[v].indexInPQ = -1;
        }
    }

    /* Batch forms (no counterpart): n pairs / n source sets per launch. */
    void SolveSSSDBatch(int32_t n, const int32_t* s, const int32_t* t, double* dist) {
        need_graph();
        check(svg_sssd_batch(g_, n, s, t, dist));
    }
    void SolveMSADBatch(int32_t n, const int64_t* set_offsets, const int32_t* srcs, const double* weights,
                        double* dist, int32_t* src_id) {
        need_graph();
        check(svg_msad_batch(g_, n, set_offsets, srcs, weights, dist, src_id));
    }

    svg_build_stats Stats() const {
        svg_build_stats st{};
        if (g_) check(svg_graph_stats(g_, &st));
        return st;
    }
    svg_build_opts& Options() { return opts_; }
    svg_graph* handle() const { return g_; }

public:
    Mesh *mesh = nullptr, *d_mesh = nullptr;
    unsigned splitInfoCoef = 10;
    unsigned vertInfoCoef = 2;
    SEARCHTYPE searchType = ASTAR;
    int K = 0;

private:
    svg_mesh* mesh_handle() const {
        svg_mesh* h = d_mesh && d_mesh->handle() ? d_mesh->handle() : (mesh ? mesh->handle() : nullptr);
        if (!h) throw Error(SVG_ERR_STATE, "AssignMesh first (a loaded mesh)");
        return h;
    }
    void need_graph() const {
        if (!g_) throw Error(SVG_ERR_STATE, "no SVG: call ConstructSVG or LoadSVGFromFile first");
    }
    svg_build_opts opts_{};
    svg_graph* g_ = nullptr;
    std::vector<int64_t> off_;
    std::vector<SVGNode> nodes_;
};

}  // namespace svg_b200

#ifndef SVG_B200_NO_GLOBAL_NAMES
using svg_b200::Edge;
using svg_b200::Face;
using svg_b200::Mesh;
using svg_b200::PriorityQueuesWithHandle;
using svg_b200::SVG;
using svg_b200::Vector3D;
using svg_b200::Vertex;
#endif

#endif
