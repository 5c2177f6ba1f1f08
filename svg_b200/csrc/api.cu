// C ABI of svg_b200 (include/svg_b200.h): object lifetime, errors, I/O.
#include <cfloat>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <unordered_map>

#include "engine.h"
#include "ich.cuh"

namespace svgb {

namespace {
thread_local std::string t_err;
cudaStream_t g_stream = nullptr;
cudaEvent_t g_mark = nullptr;
}  // namespace

void set_error(const std::string& msg) { t_err = msg; }

cudaStream_t lib_stream() {
    // created once, whichever thread asks first (a serving loop's threads and the caller's)
    static std::once_flag once;
    static cudaError_t err = cudaSuccess;
    std::call_once(once, [] { err = cudaStreamCreateWithFlags(&g_stream, cudaStreamNonBlocking); });
    if (err != cudaSuccess) throw CudaFail{err, "cudaStreamCreateWithFlags(library stream)"};
    return g_stream;
}

namespace {
struct Pool {
    std::mutex mu;
    std::multimap<size_t, void*> free_blocks;      // size -> block
    std::unordered_map<void*, size_t> live;        // block -> size
    size_t cached = 0;
    size_t in_use = 0, peak = 0;                   // bytes of live blocks, high-water mark
};
Pool& pool() {
    static Pool* P = new Pool();  // never destroyed: blocks may be freed during process exit
    return *P;
}
size_t round_block(size_t n) {
    if (n < 16) n = 16;
    if (n >= ((size_t)1 << 20)) return (n + ((size_t)2 << 20) - 1) / ((size_t)2 << 20) * ((size_t)2 << 20);
    size_t b = 512;
    while (b < n) b <<= 1;
    return b;
}
}  // namespace

void* dev_alloc(size_t bytes) {
    Pool& P = pool();
    const size_t n = round_block(bytes);
    {
        std::lock_guard<std::mutex> lk(P.mu);
        auto it = P.free_blocks.lower_bound(n);
        if (it != P.free_blocks.end() && it->first <= 2 * n) {  // reuse, wasting at most half
            void* q = it->second;
            size_t sz = it->first;
            P.free_blocks.erase(it);
            P.cached -= sz;
            P.live[q] = sz;
            P.in_use += sz;
            P.peak = std::max(P.peak, P.in_use);
            return q;
        }
    }
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, n);
    if (e != cudaSuccess) {
        cudaGetLastError();
        dev_trim();
        e = cudaMalloc(&q, n);
        if (e != cudaSuccess) {
            cudaGetLastError();
            throw SvgError{SVG_ERR_NOMEM, "device allocation of " + std::to_string(n) + " bytes failed: " +
                                              cudaGetErrorString(e)};
        }
    }
    std::lock_guard<std::mutex> lk(P.mu);
    P.live[q] = n;
    P.in_use += n;
    P.peak = std::max(P.peak, P.in_use);
    return q;
}

void dev_free(void* q) {
    if (!q) return;
    Pool& P = pool();
    if (g_stream) cudaStreamSynchronize(g_stream);  // no kernel of the library still reads it
    std::lock_guard<std::mutex> lk(P.mu);
    auto it = P.live.find(q);
    if (it == P.live.end()) return;
    P.free_blocks.emplace(it->second, q);
    P.cached += it->second;
    P.in_use -= it->second;
    P.live.erase(it);
}

void dev_usage(size_t* in_use, size_t* peak, size_t* cached, bool reset_peak) {
    Pool& P = pool();
    std::lock_guard<std::mutex> lk(P.mu);
    if (reset_peak) P.peak = P.in_use;
    if (in_use) *in_use = P.in_use;
    if (peak) *peak = P.peak;
    if (cached) *cached = P.cached;
}

size_t dev_trim() {
    Pool& P = pool();
    std::lock_guard<std::mutex> lk(P.mu);
    size_t n = 0;
    for (auto& kv : P.free_blocks) {
        cudaFree(kv.second);
        n += kv.first;
    }
    P.free_blocks.clear();
    P.cached = 0;
    return n;
}

void DevBuf::reserve(size_t n) {
    if (n <= bytes && p) return;
    release();
    if (n == 0) n = 16;
    p = dev_alloc(n);
    bytes = n;
}

void DevBuf::release() {
    if (p) dev_free(p);
    p = nullptr;
    bytes = 0;
}

DevMesh MeshDev::view() const {
    DevMesh v{};
    v.nv = nv;
    v.nf = nf;
    v.ne = ne;
    v.he = he;
    v.geo = geo;
    v.vr = vr;
    v.pos = pos;
    return v;
}

void upload_mesh(svg_mesh* m) {
    if (m->d.uploaded) return;
    const HostMesh& H = m->h;
    cudaStream_t st = lib_stream();
    MeshDev& D = m->d;
    auto al256 = [](size_t x) { return (x + 255) / 256 * 256; };
    // one block, half-edge records first: the records a window step reads
    // form one contiguous range (an L2 access-policy window can cover it)
    const size_t b_he = al256(sizeof(HeRec) * (size_t)H.ne), b_geo = al256(sizeof(HeGeo) * (size_t)H.ne),
                 b_vr = al256(sizeof(VertRec) * (size_t)H.nv), b_pos = al256(sizeof(double) * 3 * (size_t)H.nv);
    char* blk = static_cast<char*>(dev_alloc(b_he + b_geo + b_vr + b_pos));
    D.block = blk;
    D.block_bytes = b_he + b_geo + b_vr + b_pos;
    D.he = reinterpret_cast<HeRec*>(blk);
    D.geo = reinterpret_cast<HeGeo*>(blk + b_he);
    D.vr = reinterpret_cast<VertRec*>(blk + b_he + b_geo);
    D.pos = reinterpret_cast<double*>(blk + b_he + b_geo + b_vr);
    SVG_CUDA(cudaMemcpyAsync(D.he, H.he.data(), sizeof(HeRec) * (size_t)H.ne, cudaMemcpyHostToDevice, st));
    SVG_CUDA(cudaMemcpyAsync(D.geo, H.geo.data(), sizeof(HeGeo) * (size_t)H.ne, cudaMemcpyHostToDevice, st));
    SVG_CUDA(cudaMemcpyAsync(D.vr, H.vr.data(), sizeof(VertRec) * (size_t)H.nv, cudaMemcpyHostToDevice, st));
    SVG_CUDA(cudaMemcpyAsync(D.pos, H.pos.data(), sizeof(double) * 3 * (size_t)H.nv, cudaMemcpyHostToDevice, st));
    SVG_CUDA(cudaStreamSynchronize(st));
    D.nv = H.nv;
    D.nf = H.nf;
    D.ne = H.ne;
    D.uploaded = true;
}

void free_graph_device(svg_graph* g) {
    if (!g) return;
    dev_free(g->off);
    dev_free(g->adj);
    dev_free(g->dist);
    dev_free(g->paths);
    dev_free(g->st_windows);
    g->off = nullptr;
    g->adj = nullptr;
    g->dist = nullptr;
    g->paths = nullptr;
    g->st_windows = g->st_maxq = g->st_flags = nullptr;
    if (g->qdefault) qctx_free(g->qdefault);
    g->qdefault = nullptr;
}

// FP64 pipe rate: every thread runs 8 independent chains of fused
// multiply-adds (explicit __fma_rn: the library is built with --fmad=false),
// so the pipe, not latency, bounds it.
__global__ void k_dfma_rate(double* out, int iters, double b, double c) {
    double a[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) a[j] = (double)(threadIdx.x + j) * 1e-3;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int j = 0; j < 8; ++j) a[j] = __fma_rn(a[j], b, c);
    }
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < 8; ++j) s += a[j];
    if (s == 12345.678) out[0] = s;  // keeps the chains live; never true for these inputs
}

}  // namespace svgb

using namespace svgb;

// Run f, turning library exceptions into a status + svg_last_error().
template <class F>
static svg_status guarded(F&& f) {
    try {
        t_err.clear();
        return f();
    } catch (const SvgError& e) {
        set_error(e.msg);
        return e.code;
    } catch (const CudaFail& e) {
        cudaGetLastError();
        set_error(std::string("CUDA error ") + cudaGetErrorName(e.err) + " (" + cudaGetErrorString(e.err) + ") in " +
                  e.where);
        return SVG_ERR_CUDA;
    } catch (const std::bad_alloc&) {
        set_error("host allocation failed");
        return SVG_ERR_NOMEM;
    }
}

extern "C" {

const char* svg_last_error(void) { return t_err.c_str(); }

const char* svg_version(void) { return "svg_b200 0.1 (sm_100a)"; }

svg_status svg_mesh_from_arrays(int32_t nv, const double* pos, int32_t nf, const int32_t* faces, svg_mesh** out) {
    return guarded([&]() -> svg_status {
        if (!out || (!pos && nv > 0) || (!faces && nf > 0)) throw SvgError{SVG_ERR_ARG, "null argument"};
        *out = nullptr;
        svg_mesh* m = new svg_mesh();
        std::string err = build_host_mesh(nv, pos, nf, faces, m->h);
        if (!err.empty()) {
            delete m;
            throw SvgError{SVG_ERR_MESH, err};
        }
        *out = m;
        return SVG_OK;
    });
}

svg_status svg_mesh_load_obj(const char* path, svg_mesh** out) {
    return guarded([&]() -> svg_status {
        if (!path || !out) throw SvgError{SVG_ERR_ARG, "null argument"};
        *out = nullptr;
        std::vector<double> pos;
        std::vector<int32_t> faces;
        bool io = false;
        std::string err = parse_obj(path, pos, faces, io);
        if (io) throw SvgError{SVG_ERR_IO, err};
        if (!err.empty()) throw SvgError{SVG_ERR_MESH, err};
        svg_mesh* m = new svg_mesh();
        err = build_host_mesh((int32_t)(pos.size() / 3), pos.data(), (int32_t)(faces.size() / 3), faces.data(), m->h);
        if (!err.empty()) {
            delete m;
            throw SvgError{SVG_ERR_MESH, err};
        }
        *out = m;
        return SVG_OK;
    });
}

svg_status svg_mesh_upload(svg_mesh* m) {
    return guarded([&]() -> svg_status {
        if (!m) throw SvgError{SVG_ERR_ARG, "null mesh"};
        upload_mesh(m);
        return SVG_OK;
    });
}

void svg_mesh_free(svg_mesh* m) {
    if (!m) return;
    dev_free(m->d.block);
    delete m;
}

svg_status svg_mesh_counts(const svg_mesh* m, int32_t* nv, int32_t* nf, int32_t* ne) {
    if (!m) {
        set_error("null mesh");
        return SVG_ERR_ARG;
    }
    if (nv) *nv = m->h.nv;
    if (nf) *nf = m->h.nf;
    if (ne) *ne = m->h.ne;
    return SVG_OK;
}

svg_status svg_mesh_export(const svg_mesh* m, int32_t* he_v0, int32_t* he_twin, double* he_len, double* pos,
                           double* angle, int32_t* first_edge) {
    if (!m) {
        set_error("null mesh");
        return SVG_ERR_ARG;
    }
    const HostMesh& H = m->h;
    for (int32_t e = 0; e < H.ne; ++e) {
        if (he_v0) he_v0[e] = H.he[e].v0;
        if (he_twin) he_twin[e] = H.he[e].twin;
        if (he_len) he_len[e] = H.he[e].len;
    }
    if (pos) std::memcpy(pos, H.pos.data(), sizeof(double) * 3 * (size_t)H.nv);
    if (angle) std::memcpy(angle, H.angle.data(), sizeof(double) * (size_t)H.nv);
    for (int32_t v = 0; v < H.nv && first_edge; ++v) first_edge[v] = H.vr[v].first;
    return SVG_OK;
}

void svg_build_opts_default(svg_build_opts* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->K = 100;
    o->split_coef = 10;   // kernel.cu:422
    o->vert_coef = 2;
    o->win_queue_cap = 1023;     // WINPQ_SIZE - 1 (SVG.cu:18)
    o->pseudo_queue_cap = 1023;  // PSEUDOWINPQ_SIZE - 1
    o->mode = SVG_BUILD_BATCHED;
    o->with_paths = 1;
    o->heavy_first = 2;  // a K/10 probe orders a fresh mesh's first build when a lane gets few sources
    o->coop_sources = 0;  // measured: no upfront cooperative share is fastest on the benchmark meshes
    o->coop_tail = 1;
}

}  // extern "C"

namespace {
// Builds share the lane-scratch arena and run one at a time (a serving loop's
// builder thread and a caller's thread may both build).
std::mutex& build_mutex() {
    static std::mutex mu;
    return mu;
}
}  // namespace

extern "C" {

svg_status svg_build(svg_mesh* m, const svg_build_opts* opts, svg_graph** out) {
    return guarded([&]() -> svg_status {
        if (!m || !opts || !out) throw SvgError{SVG_ERR_ARG, "null argument"};
        *out = nullptr;
        std::lock_guard<std::mutex> lock(build_mutex());
        svg_graph* g = new svg_graph();
        g->mesh = m;
        try {
            run_build(m, *opts, g);
        } catch (...) {
            free_graph_device(g);
            delete g;
            throw;
        }
        *out = g;
        return SVG_OK;
    });
}

svg_status svg_build_autotune(svg_mesh* m, const svg_build_opts* opts, int32_t max_trials, svg_build_opts* best,
                              double* best_ms) {
    return guarded([&]() -> svg_status {
        if (!m || !opts) throw SvgError{SVG_ERR_ARG, "null argument"};
        std::lock_guard<std::mutex> lk(build_mutex());
        return run_autotune(m, *opts, max_trials, best, best_ms);
    });
}

svg_status svg_graph_stats(const svg_graph* g, svg_build_stats* st) {
    if (!g || !st) {
        set_error("null argument");
        return SVG_ERR_ARG;
    }
    *st = g->stats;
    return SVG_OK;
}

svg_status svg_graph_source_stats(const svg_graph* g, int32_t* windows, int32_t* max_queue, int32_t* flags) {
    return guarded([&]() -> svg_status {
        if (!g) throw SvgError{SVG_ERR_ARG, "null graph"};
        if (!g->st_windows) throw SvgError{SVG_ERR_STATE, "graph has no build statistics (loaded from file)"};
        size_t n = (size_t)g->nv * sizeof(int32_t);
        if (windows) SVG_CUDA(cudaMemcpy(windows, g->st_windows, n, cudaMemcpyDeviceToHost));
        if (max_queue) SVG_CUDA(cudaMemcpy(max_queue, g->st_maxq, n, cudaMemcpyDeviceToHost));
        if (flags) SVG_CUDA(cudaMemcpy(flags, g->st_flags, n, cudaMemcpyDeviceToHost));
        return SVG_OK;
    });
}

void svg_graph_free(svg_graph* g) {
    if (!g) return;
    free_graph_device(g);
    delete g;
}

svg_status svg_graph_counts(const svg_graph* g, int32_t* nv, int64_t* nnz, int32_t* K) {
    if (!g) {
        set_error("null graph");
        return SVG_ERR_ARG;
    }
    if (nv) *nv = g->nv;
    if (nnz) *nnz = g->nnz;
    if (K) *K = g->K;
    return SVG_OK;
}

svg_status svg_graph_copy_csr(const svg_graph* g, int64_t* offsets, int32_t* adj, double* dist) {
    return guarded([&]() -> svg_status {
        if (!g) throw SvgError{SVG_ERR_ARG, "null graph"};
        cudaStream_t st = lib_stream();
        if (offsets)
            SVG_CUDA(cudaMemcpyAsync(offsets, g->off, sizeof(int64_t) * ((size_t)g->nv + 1), cudaMemcpyDeviceToHost, st));
        if (adj && g->nnz)
            SVG_CUDA(cudaMemcpyAsync(adj, g->adj, sizeof(int32_t) * (size_t)g->nnz, cudaMemcpyDeviceToHost, st));
        if (dist && g->nnz)
            SVG_CUDA(cudaMemcpyAsync(dist, g->dist, sizeof(double) * (size_t)g->nnz, cudaMemcpyDeviceToHost, st));
        SVG_CUDA(cudaStreamSynchronize(st));
        return SVG_OK;
    });
}

svg_status svg_graph_copy_nodes(const svg_graph* g, int32_t* tails, svg_node* nodes) {
    return guarded([&]() -> svg_status {
        if (!g) throw SvgError{SVG_ERR_ARG, "null graph"};
        std::vector<int64_t> off((size_t)g->nv + 1);
        std::vector<int32_t> adj((size_t)g->nnz);
        std::vector<double> dist((size_t)g->nnz);
        std::vector<PathEnd> pe(g->with_paths ? (size_t)g->nnz : 0);
        cudaStream_t st = lib_stream();
        SVG_CUDA(cudaMemcpyAsync(off.data(), g->off, sizeof(int64_t) * off.size(), cudaMemcpyDeviceToHost, st));
        if (g->nnz) {
            SVG_CUDA(cudaMemcpyAsync(adj.data(), g->adj, sizeof(int32_t) * adj.size(), cudaMemcpyDeviceToHost, st));
            SVG_CUDA(cudaMemcpyAsync(dist.data(), g->dist, sizeof(double) * dist.size(), cudaMemcpyDeviceToHost, st));
            if (g->with_paths)
                SVG_CUDA(cudaMemcpyAsync(pe.data(), g->paths, sizeof(PathEnd) * pe.size(), cudaMemcpyDeviceToHost, st));
        }
        SVG_CUDA(cudaStreamSynchronize(st));
        for (int32_t v = 0; v < g->nv && tails; ++v) tails[v] = (int32_t)(off[v + 1] - off[v]);
        for (int64_t i = 0; i < g->nnz && nodes; ++i) {
            svg_node& n = nodes[i];
            n.adj = adj[i];
            n.pad_ = 0;
            n.dist = dist[i];
            if (g->with_paths) {
                n.next_to_src_edge = pe[i].src_edge;
                n.next_to_dst_edge = pe[i].dst_edge;
                n.next_to_src_x = pe[i].src_x;
                n.next_to_dst_x = pe[i].dst_x;
            } else {
                n.next_to_src_edge = n.next_to_dst_edge = 0xFFFFFFFFu;
                n.next_to_src_x = n.next_to_dst_x = 0.0;
            }
        }
        return SVG_OK;
    });
}

svg_status svg_graph_device_csr(const svg_graph* g, const int64_t** offsets, const int32_t** adj, const double** dist) {
    if (!g) {
        set_error("null graph");
        return SVG_ERR_ARG;
    }
    if (offsets) *offsets = g->off;
    if (adj) *adj = g->adj;
    if (dist) *dist = g->dist;
    return SVG_OK;
}

// SVG::SaveSVGToFile (SVG.cu:208-217): per vertex int32 degree + degree SVGNodes.
svg_status svg_graph_save(const svg_graph* g, const char* path) {
    return guarded([&]() -> svg_status {
        if (!g || !path) throw SvgError{SVG_ERR_ARG, "null argument"};
        std::vector<int32_t> tails((size_t)g->nv);
        std::vector<svg_node> nodes((size_t)g->nnz);
        svg_status s = svg_graph_copy_nodes(g, tails.data(), nodes.data());
        if (s != SVG_OK) return s;
        FILE* f = std::fopen(path, "wb");
        if (!f) throw SvgError{SVG_ERR_IO, std::string("cannot open ") + path + " for writing"};
        size_t k = 0;
        bool ok = true;
        for (int32_t v = 0; v < g->nv && ok; ++v) {
            ok = std::fwrite(&tails[v], sizeof(int32_t), 1, f) == 1;
            if (ok && tails[v]) ok = std::fwrite(&nodes[k], sizeof(svg_node), (size_t)tails[v], f) == (size_t)tails[v];
            k += (size_t)tails[v];
        }
        if (std::fclose(f) != 0) ok = false;
        if (!ok) throw SvgError{SVG_ERR_IO, std::string("short write to ") + path};
        return SVG_OK;
    });
}

// SVG::LoadSVGFromFile (SVG.cu:219-239).  Rows longer than K are rejected
// (the reference would overrun its V*K array).
svg_status svg_graph_load(svg_mesh* m, int32_t K, const char* path, svg_graph** out) {
    return guarded([&]() -> svg_status {
        if (!m || !path || !out || K <= 0) throw SvgError{SVG_ERR_ARG, "bad argument"};
        *out = nullptr;
        FILE* f = std::fopen(path, "rb");
        if (!f) throw SvgError{SVG_ERR_IO, std::string("cannot open file ") + path};
        const int32_t nv = m->h.nv;
        std::vector<int64_t> off((size_t)nv + 1, 0);
        std::vector<svg_node> nodes;
        nodes.reserve((size_t)nv * 8);
        for (int32_t v = 0; v < nv; ++v) {
            int32_t d = 0;
            if (std::fread(&d, sizeof(int32_t), 1, f) != 1 || d < 0 || d > K) {
                std::fclose(f);
                throw SvgError{SVG_ERR_IO, "bad or truncated row " + std::to_string(v) + " in " + path};
            }
            size_t b = nodes.size();
            nodes.resize(b + (size_t)d);
            if (d && std::fread(&nodes[b], sizeof(svg_node), (size_t)d, f) != (size_t)d) {
                std::fclose(f);
                throw SvgError{SVG_ERR_IO, "truncated row " + std::to_string(v) + " in " + path};
            }
            off[v + 1] = off[v] + d;
        }
        std::fclose(f);
        upload_mesh(m);
        svg_graph* g = new svg_graph();
        g->mesh = m;
        g->K = K;
        g->nv = nv;
        g->nnz = (int64_t)nodes.size();
        g->with_paths = true;
        try {
            std::vector<int32_t> adj(nodes.size());
            std::vector<double> dist(nodes.size());
            std::vector<PathEnd> pe(nodes.size());
            for (size_t i = 0; i < nodes.size(); ++i) {
                if (nodes[i].adj < 0 || nodes[i].adj >= nv) throw SvgError{SVG_ERR_IO, "vertex id out of range in file"};
                adj[i] = nodes[i].adj;
                dist[i] = nodes[i].dist;
                pe[i] = PathEnd{nodes[i].next_to_src_edge, nodes[i].next_to_dst_edge, nodes[i].next_to_src_x,
                                nodes[i].next_to_dst_x};
            }
            size_t E = std::max<size_t>(nodes.size(), 1);
            g->off = dev_alloc_n<int64_t>(off.size());
            g->adj = dev_alloc_n<int32_t>(E);
            g->dist = dev_alloc_n<double>(E);
            g->paths = dev_alloc(sizeof(PathEnd) * E);
            SVG_CUDA(cudaMemcpy(g->off, off.data(), sizeof(int64_t) * off.size(), cudaMemcpyHostToDevice));
            if (!nodes.empty()) {
                SVG_CUDA(cudaMemcpy(g->adj, adj.data(), sizeof(int32_t) * adj.size(), cudaMemcpyHostToDevice));
                SVG_CUDA(cudaMemcpy(g->dist, dist.data(), sizeof(double) * dist.size(), cudaMemcpyHostToDevice));
                SVG_CUDA(cudaMemcpy(g->paths, pe.data(), sizeof(PathEnd) * pe.size(), cudaMemcpyHostToDevice));
            }
        } catch (...) {
            free_graph_device(g);
            delete g;
            throw;
        }
        *out = g;
        return SVG_OK;
    });
}

svg_status svg_sssd_batch_device(svg_graph* g, int32_t n, const int32_t* d_s, const int32_t* d_t, double* d_dist) {
    return guarded([&]() -> svg_status {
        if (!g || n < 0 || (n > 0 && (!d_s || !d_t || !d_dist))) throw SvgError{SVG_ERR_ARG, "bad argument"};
        return run_sssd(g, n, d_s, d_t, d_dist);
    });
}

svg_status svg_msad_batch_device(svg_graph* g, int32_t n, const int64_t* d_set_offsets, const int32_t* d_srcs,
                                 const double* d_weights, double* d_dist, int32_t* d_src_id) {
    return guarded([&]() -> svg_status {
        if (!g || n < 0 || (n > 0 && (!d_set_offsets || !d_dist))) throw SvgError{SVG_ERR_ARG, "bad argument"};
        return run_msad(g, n, d_set_offsets, d_srcs, d_weights, d_dist, d_src_id, -1);
    });
}

svg_status svg_graph_set_query_form(svg_graph* g, int32_t form) {
    return guarded([&]() -> svg_status {
        if (!g || (form != SVG_QUERY_CLUSTER && form != SVG_QUERY_PLAIN))
            throw SvgError{SVG_ERR_ARG, "bad argument"};
        if (g->qform != form && g->qdefault) {
            SVG_CUDA(cudaStreamSynchronize(lib_stream()));
            qctx_free(g->qdefault);
            g->qdefault = nullptr;
        }
        g->qform = form;
        return SVG_OK;
    });
}

svg_status svg_sssd_batch(svg_graph* g, int32_t n, const int32_t* s, const int32_t* t, double* dist) {
    return guarded([&]() -> svg_status {
        if (!g || n < 0 || (n > 0 && (!s || !t || !dist))) throw SvgError{SVG_ERR_ARG, "bad argument"};
        if (n == 0) return SVG_OK;
        for (int32_t i = 0; i < n; ++i)
            if (s[i] < 0 || s[i] >= g->nv || t[i] < 0 || t[i] >= g->nv)
                throw SvgError{SVG_ERR_ARG, "query vertex out of range at pair " + std::to_string(i)};
        cudaStream_t st = lib_stream();
        DevBuf b;
        b.reserve((size_t)n * (4 + 4 + 8) + 64);
        int32_t* ds = b.as<int32_t>();
        int32_t* dt = ds + n;
        double* dd = reinterpret_cast<double*>(reinterpret_cast<char*>(b.p) + (((size_t)n * 8 + 15) / 16) * 16);
        SVG_CUDA(cudaMemcpyAsync(ds, s, sizeof(int32_t) * n, cudaMemcpyHostToDevice, st));
        SVG_CUDA(cudaMemcpyAsync(dt, t, sizeof(int32_t) * n, cudaMemcpyHostToDevice, st));
        svg_status r = run_sssd(g, n, ds, dt, dd);
        if (r != SVG_OK) return r;
        SVG_CUDA(cudaMemcpyAsync(dist, dd, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
        SVG_CUDA(cudaStreamSynchronize(st));
        return SVG_OK;
    });
}

}  // extern "C"

namespace {
// svg_msad_batch and svg_msad_batch_paths: host buffers in and out; parent
// pointers (optional) from the finished distances on the device.
svg_status msad_host(svg_graph* g, int32_t n, const int64_t* set_offsets, const int32_t* srcs, const double* weights,
                     double* dist, int32_t* src_id, int32_t* parent) {
    if (!g || n < 0 || (n > 0 && (!set_offsets || !dist))) throw SvgError{SVG_ERR_ARG, "bad argument"};
    if (n == 0) return SVG_OK;
    int64_t total = set_offsets[n];
    if (set_offsets[0] != 0 || total < 0) throw SvgError{SVG_ERR_ARG, "set_offsets must start at 0"};
    for (int32_t q = 0; q < n; ++q)
        if (set_offsets[q + 1] < set_offsets[q]) throw SvgError{SVG_ERR_ARG, "set_offsets not monotone"};
    if (total > 0 && (!srcs || !weights)) throw SvgError{SVG_ERR_ARG, "null sources"};
    for (int64_t i = 0; i < total; ++i)
        if (srcs[i] < 0 || srcs[i] >= g->nv) throw SvgError{SVG_ERR_ARG, "source vertex out of range"};
    cudaStream_t st = lib_stream();
    DevBuf b;
    const bool want_src = src_id || parent;  // a source keeps parent -1 only where it kept its own label
    size_t ob = sizeof(int64_t) * ((size_t)n + 1), sb = sizeof(int32_t) * (size_t)std::max<int64_t>(total, 1),
           wb = sizeof(double) * (size_t)std::max<int64_t>(total, 1), db = sizeof(double) * (size_t)n * g->nv,
           ib = want_src ? sizeof(int32_t) * (size_t)n * g->nv : 0, pb = parent ? sizeof(int32_t) * (size_t)n * g->nv : 0;
    auto al = [](size_t x) { return (x + 255) / 256 * 256; };
    b.reserve(al(ob) + al(sb) + al(wb) + al(db) + al(ib) + al(pb) + 256);
    char* p = b.as<char>();
    int64_t* doff = reinterpret_cast<int64_t*>(p); p += al(ob);
    int32_t* dsrc = reinterpret_cast<int32_t*>(p); p += al(sb);
    double* dw = reinterpret_cast<double*>(p); p += al(wb);
    double* dd = reinterpret_cast<double*>(p); p += al(db);
    int32_t* did = want_src ? reinterpret_cast<int32_t*>(p) : nullptr; p += al(ib);
    int32_t* dpar = parent ? reinterpret_cast<int32_t*>(p) : nullptr;
    SVG_CUDA(cudaMemcpyAsync(doff, set_offsets, ob, cudaMemcpyHostToDevice, st));
    if (total > 0) {
        SVG_CUDA(cudaMemcpyAsync(dsrc, srcs, sizeof(int32_t) * total, cudaMemcpyHostToDevice, st));
        SVG_CUDA(cudaMemcpyAsync(dw, weights, sizeof(double) * total, cudaMemcpyHostToDevice, st));
    }
    svg_status r = run_msad(g, n, doff, dsrc, dw, dd, did, total);
    if (r != SVG_OK) return r;
    if (dpar) query_parents(g, n, dd, did, dpar, st);
    SVG_CUDA(cudaMemcpyAsync(dist, dd, db, cudaMemcpyDeviceToHost, st));
    if (src_id) SVG_CUDA(cudaMemcpyAsync(src_id, did, ib, cudaMemcpyDeviceToHost, st));
    if (parent) SVG_CUDA(cudaMemcpyAsync(parent, dpar, pb, cudaMemcpyDeviceToHost, st));
    SVG_CUDA(cudaStreamSynchronize(st));
    return SVG_OK;
}
}  // namespace

extern "C" {

svg_status svg_msad_batch(svg_graph* g, int32_t n, const int64_t* set_offsets, const int32_t* srcs,
                          const double* weights, double* dist, int32_t* src_id) {
    return guarded([&]() -> svg_status { return msad_host(g, n, set_offsets, srcs, weights, dist, src_id, nullptr); });
}

svg_status svg_msad_batch_paths(svg_graph* g, int32_t n, const int64_t* set_offsets, const int32_t* srcs,
                                const double* weights, double* dist, int32_t* src_id, int32_t* parent) {
    return guarded([&]() -> svg_status {
        if (!parent) throw SvgError{SVG_ERR_ARG, "parent buffer is null"};
        return msad_host(g, n, set_offsets, srcs, weights, dist, src_id, parent);
    });
}

svg_status svg_sssd_path(svg_graph* g, int32_t s, int32_t t, int32_t cap, int32_t* path, double* path_dist,
                         int32_t* len, double* dist) {
    return guarded([&]() -> svg_status {
        if (!g || !len || cap < 0 || (cap > 0 && !path)) throw SvgError{SVG_ERR_ARG, "bad argument"};
        if (s < 0 || s >= g->nv || t < 0 || t >= g->nv) throw SvgError{SVG_ERR_ARG, "query vertex out of range"};
        const size_t V = (size_t)g->nv;
        std::vector<double> d(V);
        std::vector<int32_t> par(V);
        const int64_t off[2] = {0, 1};
        const double w0 = 0.0;
        svg_status r = msad_host(g, 1, off, &s, &w0, d.data(), nullptr, par.data());
        if (r != SVG_OK) return r;
        if (dist) *dist = d[(size_t)t];
        *len = 0;
        if (!(d[(size_t)t] < DBL_MAX)) return SVG_OK;  // unreachable: empty path
        if (d[(size_t)t] < 0.0) throw SvgError{SVG_ERR_NOMEM, "the search exceeded its round limit"};
        int32_t n = 0;
        for (int32_t v = t;; v = par[(size_t)v]) {
            if (v < 0 || n > g->nv) throw SvgError{SVG_ERR_STATE, "parent chain does not reach the source"};
            if (n < cap) {
                path[n] = v;
                if (path_dist) path_dist[n] = d[(size_t)v];
            }
            ++n;
            if (v == s) break;
        }
        *len = n;
        if (n > cap) throw SvgError{SVG_ERR_ARG, "path has " + std::to_string(n) + " vertices, cap " + std::to_string(cap)};
        return SVG_OK;
    });
}

size_t svg_trim_device_cache(void) { return dev_trim(); }

void svg_device_memory(int64_t* in_use, int64_t* peak, int64_t* cached, int32_t reset_peak) {
    size_t a = 0, b = 0, c = 0;
    dev_usage(&a, &b, &c, reset_peak != 0);
    if (in_use) *in_use = (int64_t)a;
    if (peak) *peak = (int64_t)b;
    if (cached) *cached = (int64_t)c;
}

svg_status svg_device_fp64_rate(double* fma_per_s) {
    return guarded([&]() -> svg_status {
        if (!fma_per_s) throw SvgError{SVG_ERR_ARG, "null argument"};
        int dev = 0, sms = 0;
        SVG_CUDA(cudaGetDevice(&dev));
        SVG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        cudaStream_t st = lib_stream();
        double* d = dev_alloc_n<double>(1);
        const int blocks = sms * 8, threads = 256, iters = 1 << 14;
        cudaEvent_t e0, e1;
        SVG_CUDA(cudaEventCreate(&e0));
        SVG_CUDA(cudaEventCreate(&e1));
        k_dfma_rate<<<blocks, threads, 0, st>>>(d, 256, 0.999999, 1e-7);  // warm-up
        SVG_CUDA(cudaEventRecord(e0, st));
        k_dfma_rate<<<blocks, threads, 0, st>>>(d, iters, 0.999999, 1e-7);
        SVG_CUDA(cudaEventRecord(e1, st));
        SVG_CUDA(cudaEventSynchronize(e1));
        SVG_CUDA(cudaGetLastError());
        float ms = 0.f;
        SVG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        dev_free(d);
        *fma_per_s = (double)blocks * threads * 8.0 * iters / (ms / 1e3);
        return SVG_OK;
    });
}

svg_status svg_timer_mark(double* ms_since_last) {
    return guarded([&]() -> svg_status {
        cudaStream_t st = lib_stream();
        cudaEvent_t e;
        SVG_CUDA(cudaEventCreate(&e));
        SVG_CUDA(cudaEventRecord(e, st));
        SVG_CUDA(cudaEventSynchronize(e));
        double ms = 0.0;
        if (g_mark) {
            float f = 0.f;
            SVG_CUDA(cudaEventElapsedTime(&f, g_mark, e));
            ms = f;
            cudaEventDestroy(g_mark);
        }
        g_mark = e;
        if (ms_since_last) *ms_since_last = ms;
        return SVG_OK;
    });
}

}  // extern "C"
