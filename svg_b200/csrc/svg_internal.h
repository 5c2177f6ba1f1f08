// Internal types shared by the host library and the CUDA kernels.
#pragma once

#include <cstdint>
#include <string>
#include <memory>
#include <utility>
#include <vector>

#include "svg_b200.h"

namespace svgb {

// Half-edge record, 32 bytes: one sector.  Half-edge e belongs to face e/3;
// next(e) and prev(e) are arithmetic (3f + (j+1)%3, 3f + (j+2)%3) exactly as
// the reference numbers them (Mesh.cu:73-74), so they are not stored.
struct alignas(32) HeRec {
    int32_t v0;      // edges[e].verts[0]
    int32_t v1;      // edges[e].verts[1]
    int32_t twin;    // -1 on the boundary
    int32_t pad;
    double len;      // edges[e].edgeLen
    double corner;   // corner angle of face(e) at v0(e): acos of the law of cosines, clamped
};

// Per-half-edge planar unfolding of face(e) onto e's line (e from (0,0) to (len,0)):
//   apex = third vertex below the line, as PropagateWindow builds it (ICHDevice.cu:632-634)
//   top  = third vertex above the line measured for the window on e (IsValidWindow, :916-918)
struct alignas(32) HeGeo {
    double ax, ay;
    double tx, ty;
};

enum : int32_t { kVertSaddleGE = 1, kVertSaddleGT = 2 };  // angle >= 2pi, angle > 2pi

struct VertRec {
    int32_t first;   // firstEdge: last half-edge leaving the vertex (Mesh.cu:121)
    int32_t flags;
};

struct DevMesh {
    int32_t nv, nf, ne;
    const HeRec* he;
    const HeGeo* geo;
    const VertRec* vr;
    const double* pos;
};

// Host half-edge construction (Mesh::LoadFromFile semantics).
// Allocator whose resize() leaves new elements uninitialised: the mesh build
// writes every element in parallel loops, so the pages are first touched (and
// faulted in) by many threads instead of by one zero-filling pass.
template <class T>
struct UninitAlloc : std::allocator<T> {
    template <class U>
    struct rebind {
        using other = UninitAlloc<U>;
    };
    UninitAlloc() = default;
    template <class U>
    UninitAlloc(const UninitAlloc<U>&) {}
    template <class U>
    void construct(U* p) {
        ::new (static_cast<void*>(p)) U;
    }
    template <class U, class... A>
    void construct(U* p, A&&... a) {
        ::new (static_cast<void*>(p)) U(std::forward<A>(a)...);
    }
};

struct HostMesh {
    int32_t nv = 0, nf = 0, ne = 0;
    std::vector<double> pos;      // 3*nv
    std::vector<int32_t> faces;   // 3*nf
    std::vector<HeRec, UninitAlloc<HeRec>> he;
    std::vector<HeGeo, UninitAlloc<HeGeo>> geo;
    std::vector<VertRec> vr;
    std::vector<double> angle;
};

// Returns an empty string on success, else the reason.
std::string build_host_mesh(int32_t nv, const double* pos, int32_t nf, const int32_t* faces, HostMesh& m);
std::string parse_obj(const char* path, std::vector<double>& pos, std::vector<int32_t>& faces, bool& io_error);

}  // namespace svgb
