// Library objects and host-side helpers shared by the C-ABI and the kernels' launchers.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "svg_b200.h"
#include "svg_internal.h"

namespace svgb {

struct BuildGraph;  // a build captured as a CUDA graph (build.cu)

void set_error(const std::string& msg);

struct CudaFail {
    cudaError_t err;
    std::string where;
};

#define SVG_CUDA(call)                                                                      \
    do {                                                                                    \
        cudaError_t e__ = (call);                                                           \
        if (e__ != cudaSuccess) throw ::svgb::CudaFail{e__, std::string(#call) + " @ " + __FILE__ + ":" + std::to_string(__LINE__)}; \
    } while (0)

struct SvgError {
    svg_status code;
    std::string msg;
};

// The library's CUDA stream and events (one device: the current one at first use).
cudaStream_t lib_stream();

// Device memory through a caching pool: freed blocks are kept by size and
// handed out again, so repeated builds and query batches do not pay for
// cudaMalloc/cudaFree of gigabyte buffers.  dev_free waits for the library
// stream before a block can be reused.  A failing cudaMalloc releases the
// cached blocks and retries once.
void* dev_alloc(size_t bytes);
void dev_free(void* p);
size_t dev_trim();  // release every cached block; returns the bytes released
// bytes of live blocks, their high-water mark, bytes cached for reuse
void dev_usage(size_t* in_use, size_t* peak, size_t* cached, bool reset_peak);
template <class T> T* dev_alloc_n(size_t n) { return static_cast<T*>(dev_alloc(n * sizeof(T))); }

// Growable device buffer, reused across calls.
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    void reserve(size_t n);   // grows (contents not preserved)
    void release();
    template <class T> T* as() const { return static_cast<T*>(p); }
    ~DevBuf() { release(); }
};

struct MeshDev {
    bool uploaded = false;
    void* block = nullptr;   // one allocation holding he, geo, vr, pos in that order
    size_t block_bytes = 0;
    int32_t nv = 0, nf = 0, ne = 0;
    HeRec* he = nullptr;
    HeGeo* geo = nullptr;
    VertRec* vr = nullptr;
    double* pos = nullptr;
    DevMesh view() const;
};

}  // namespace svgb

struct svg_mesh {
    svgb::HostMesh h;
    svgb::MeshDev d;
    // Per-source cost (windows propagated) measured by the last batched build
    // at K = cost_K: the next build at the same K orders its work queue
    // heaviest first (longest-processing-time first).
    int32_t cost_K = 0;
    std::vector<int32_t> cost;
    // the costs are a K/10 probe build's stand-in, not a build at cost_K
    bool cost_probe = false;
    // the last build captured as a CUDA graph (opts.graph), replayed by later
    // builds with the same options
    std::shared_ptr<svgb::BuildGraph> build_graph;
    // Launch parameters svg_build_autotune chose, per K.
    struct Tuned {
        int32_t K;
        svg_build_opts opts;
        double ms;
    };
    std::vector<Tuned> tuned;
};

struct svg_qctx;

struct svg_graph {
    svg_mesh* mesh = nullptr;
    int32_t K = 0;
    int32_t nv = 0;
    int64_t nnz = 0;
    bool with_paths = false;
    int64_t* off = nullptr;        // nv+1
    int32_t* adj = nullptr;        // nnz
    double* dist = nullptr;        // nnz
    void* paths = nullptr;         // nnz PathEnd (optional)
    int32_t* st_windows = nullptr; // nv per-source counters (device)
    int32_t* st_maxq = nullptr;
    int32_t* st_flags = nullptr;
    svg_build_stats stats{};
    // queries: near-far bucket width (mean edge length) and the context of
    // the synchronous batch entry points
    double delta = 0.0;
    svg_qctx* qdefault = nullptr;
    int32_t qform = SVG_QUERY_CLUSTER;  // kernel form of the synchronous query calls
};

// Scratch of `slots` concurrent queries on one graph (see query.cu).
struct svg_qctx {
    svg_graph* g = nullptr;
    int slots = 0;
    size_t slot_bytes = 0;
    int64_t list_cap = 0;
    svgb::DevBuf buf;
    uint32_t* stamps = nullptr;
    int32_t* head = nullptr;
    int cluster = 0;  // blocks per query: a cluster of them, or 0 for one block (the plain form)
    bool adaptive = false;  // large batches switch to 8-block clusters
};

namespace svgb {
svg_status run_build(svg_mesh* m, const svg_build_opts& o, svg_graph* g);
svg_status run_autotune(svg_mesh* m, const svg_build_opts& o, int32_t max_trials, svg_build_opts* best,
                        double* best_ms);
void upload_mesh(svg_mesh* m);
void free_graph_device(svg_graph* g);
svg_status run_sssd(svg_graph* g, int32_t n, const int32_t* d_s, const int32_t* d_t, double* d_dist);
svg_status run_msad(svg_graph* g, int32_t n, const int64_t* d_off, const int32_t* d_src, const double* d_w,
                    double* d_dist, int32_t* d_src_id, int64_t total_srcs);
double graph_delta(svg_graph* g, cudaStream_t st);
svg_qctx* qctx_create(svg_graph* g, int slots, cudaStream_t st, int cluster);
int query_slots_per_sm();            // plain form: query blocks resident per SM
int query_cluster_size();            // cluster form: blocks per query
int query_cluster_slots(int csize);  // cluster form: clusters resident at once
void qctx_free(svg_qctx* c);
// parent pointers of n finished MSAD searches on the device (d_src may be null)
void query_parents(svg_graph* g, int32_t n, const double* d_dist, const int32_t* d_src, int32_t* d_parent,
                   cudaStream_t st);
void qctx_sssd(svg_qctx* c, int32_t n, const int32_t* d_s, const int32_t* d_t, double* d_dist, cudaStream_t st);
void qctx_msad(svg_qctx* c, int32_t n, const int64_t* d_off, const int32_t* d_src, const double* d_w, double* d_dist,
               int32_t* d_src_id, cudaStream_t st);
}  // namespace svgb
