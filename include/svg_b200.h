/* svg_b200: B200-native Saddle Vertex Graph (SVG) geodesic engine - C ABI.
 *
 * The drop-in boundary for the reference's Mesh / SVG host classes
 * (Mesh.cuh:33-52, SVG.cuh:18-113).  Plain pointers and sizes only; every call
 * returns an svg_status, never exits, and leaves a message for
 * svg_last_error() on failure (the reference prints and exit(-1)s through
 * HANDLE_ERROR, book.cuh:23-33).  One GPU; handles are not thread-safe, like
 * the reference classes (SVG::searchType is mutable state, SVG.cu:245).
 *
 * Geometry is float64 throughout.  Vertex and half-edge ids are int32.
 * Half-edge 3f+j of face f runs from faces[3f+j] to faces[3f+(j+1)%3].
 */
#ifndef SVG_B200_H
#define SVG_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum svg_status {
    SVG_OK = 0,
    SVG_ERR_ARG = 1,      /* bad argument or size */
    SVG_ERR_IO = 2,       /* file cannot be opened / short read */
    SVG_ERR_CUDA = 3,     /* CUDA runtime error (message has the CUDA text) */
    SVG_ERR_NOMEM = 4,    /* device or host allocation failed, or over the HBM budget */
    SVG_ERR_MESH = 5,     /* mesh unusable (no faces, bad index, too large) */
    SVG_ERR_STATE = 6     /* call out of order (e.g. graph of another mesh) */
} svg_status;

typedef struct svg_mesh svg_mesh;    /* host half-edge mesh + its device copy */
typedef struct svg_graph svg_graph;  /* one built SVG, resident on the device */

/* One SVG edge in the reference's on-disk and host layout, SVG::SVGNode
 * (SVG.cuh:21-27), 40 bytes: adjacent vertex, geodesic length, and the first
 * and last key points of the geodesic (half-edge id + position along it). */
typedef struct svg_node {
    int32_t adj;
    int32_t pad_;
    double dist;
    uint32_t next_to_src_edge;
    uint32_t next_to_dst_edge;
    double next_to_src_x;
    double next_to_dst_x;
} svg_node;

/* Last error message of this thread ("" if none). */
const char* svg_last_error(void);

/* Library version string. */
const char* svg_version(void);

/* ---------------------------------------------------------------- meshes */

/* Mesh::LoadFromFile (Mesh.cu:24-126): OBJ `v x y z` and `f a b c` lines
 * (1-based), same half-edge numbering, twin pairing, vertex angle sums and
 * firstEdge as the reference.  Boundary half-edges get twin -1. */
svg_status svg_mesh_load_obj(const char* path, svg_mesh** out);

/* The same mesh from arrays: pos[3*nv] (x,y,z), faces[3*nf] (0-based). */
svg_status svg_mesh_from_arrays(int32_t nv, const double* pos, int32_t nf, const int32_t* faces,
                                svg_mesh** out);

/* Mesh::copyToGPU (Mesh.cu:128-142): upload the structure-of-arrays device
 * layout.  Builds call it implicitly; an explicit call times the upload. */
svg_status svg_mesh_upload(svg_mesh* m);

/* Mesh::clear + Mesh::clearGPU (Mesh.cu:144-158). */
void svg_mesh_free(svg_mesh* m);

svg_status svg_mesh_counts(const svg_mesh* m, int32_t* nv, int32_t* nf, int32_t* ne);

/* Host copies of the loaded structure (any pointer may be NULL): half-edge
 * start vertex, twin (-1 on the boundary), length; vertex position, angle sum,
 * firstEdge (the last half-edge leaving the vertex, -1 if isolated). */
svg_status svg_mesh_export(const svg_mesh* m, int32_t* he_v0, int32_t* he_twin, double* he_len,
                           double* pos, double* angle, int32_t* first_edge);

/* ------------------------------------------------------------------ build */

typedef enum svg_build_mode {
    SVG_BUILD_BATCHED = 0,  /* persistent kernel, device work queue, warp-cooperative emission */
    SVG_BUILD_PLAIN = 1     /* one source per thread, grid-stride, O(V) emission scan (reference form) */
} svg_build_mode;

typedef struct svg_build_opts {
    int32_t K;                /* SVG::SetParameters K (SVG.cu:114): ICH stops after K new vertices */
    uint32_t split_coef;      /* reference split hash size = K*split_coef (default 10, kernel.cu:422) */
    uint32_t vert_coef;       /* reference vertex hash size = K*vert_coef (default 2) */
    int32_t win_queue_cap;    /* window queue capacity, pushes beyond it are dropped (reference 1023) */
    int32_t pseudo_queue_cap; /* pseudo-source queue capacity (reference 1023) */
    int32_t mode;             /* svg_build_mode */
    int32_t threads_per_block;/* 0 = autotuned (batched) / 128 (plain, SVG.cuh:11) */
    int32_t blocks;           /* 0 = autotuned (batched) / 64 (plain, SVG.cuh:10) */
    int32_t with_paths;       /* 1 = also produce the path-end fields of svg_node */
    int32_t heavy_first;      /* batched: order the work queue heaviest first, by the per-source cost of the
                                 mesh's previous build at this K (1), or, lacking one, of a probe build at
                                 K/10 when K >= 160 and a launch's lanes get at most 4 sources each
                                 (2, the default); 0: vertex order */
    int64_t hbm_budget;       /* bytes of scratch the build may hold (0 = automatic) */
    int32_t source_begin;     /* build rows for sources [source_begin, source_end) only; */
    int32_t source_end;       /* 0,0 = all vertices */
    int32_t coop_sources;     /* batched, with a heaviest-first order: this many of the heaviest sources are
                                 each run by a whole warp (warp-cooperative heap and table operations), the
                                 rest one per lane; -1 automatic (those whose cost exceeds a lane's average
                                 share), 0 none (the default) */
    int32_t coop_warps;       /* warps that run them (0 automatic) */
    int32_t vote_wait;        /* batched: most loop iterations a lane waits for the warp's vote to pick its
                                 kind of step (0 = 8) */
    int32_t heavy_waves;      /* batched: waves of lanes filled heaviest-first before vertex order (0 = 2) */
    int32_t heap_factor;      /* batched: first-pass physical window heap = heap_factor x K entries (0 = 3);
                                 a source that outgrows it is re-run with the full 1023 */
    int32_t autotune;         /* batched: 1 = use the parameters svg_build_autotune cached on this mesh for
                                 this K (if any) in place of the fields above and of blocks */
    int32_t coop_tail;        /* batched: 1 (default) = once the work queue is drained, a warp left with one
                                 running lane finishes that lane's source on all 32 threads; 0 = off */
    int32_t graph;            /* batched: 1 = the build's device work (memsets, window propagation, offsets
                                 scan, emission, copies into the graph's buffers) is captured in a CUDA graph
                                 kept with the mesh, and later builds of the mesh with the same options
                                 replay it (one launch, no host round trip); a replay whose sources outgrow
                                 the captured sizes falls back to the ordinary build */
} svg_build_opts;

typedef struct svg_build_stats {
    double ms_total;          /* device time of the build, CUDA events on the build stream */
    double ms_ich;            /* window-propagation phase */
    double ms_emit;           /* edge emission (+ compaction) */
    int64_t windows;          /* windows propagated */
    int64_t windows_generated;/* windows created (reference numOfWinGen, summed) */
    int64_t pseudo_sources;   /* pseudo-sources expanded */
    int64_t edges;            /* SVG edges emitted */
    int32_t sources;
    int32_t max_win_queue;    /* queue high-water marks over all sources */
    int32_t max_pseudo_queue;
    int32_t queue_drop_sources; /* sources whose queue was full at a push (reference drops too) */
    int32_t ref_overflow_sources; /* sources where the reference's fixed hash tables overflow: results
                                     follow a map without overflow there, not the reference */
    int32_t watchdog_sources; /* sources stopped by an iteration cap (reference would spin) */
    int32_t undefined_sources;/* sources reaching a step the reference leaves undefined */
    int32_t retried_sources;  /* sources re-run with larger scratch tables */
    int32_t launches;         /* kernels launched */
    int64_t scratch_bytes;    /* device scratch held by the build */
    int32_t coop_sources;     /* sources run by whole warps */
    int32_t coop_warps;       /* warps that ran them */
    int32_t graph_replayed;   /* 1: this build was a replay of the mesh's captured graph (opts.graph) */
} svg_build_stats;

void svg_build_opts_default(svg_build_opts* o);

/* SVG::SetParameters + Allocation + ConstructSVG + Free (SVG.cu:114-182):
 * build the SVG of mesh m on the device.  The graph stays resident.  Builds
 * from several threads are safe; they run one at a time. */
svg_status svg_build(svg_mesh* m, const svg_build_opts* opts, svg_graph** out);

/* Autotuner (no counterpart in the reference): times full batched builds of
 * mesh m at opts->K with candidate launch parameters - how many of the
 * heaviest sources run on whole warps and with how many warps, blocks per SM,
 * the vote wait limit, the heavy-first waves and the physical heap factor -
 * one parameter at a time from the current best (at most max_trials builds,
 * 0 = 16), checks that every candidate builds the same graph (a checksum of
 * the CSR), and caches the fastest on the mesh for this K: later svg_build
 * calls with opts.autotune = 1 use it.  *best (optional) receives the chosen
 * options, *best_ms (optional) its build time.  The parameters change only
 * the schedule, never the graph. */
svg_status svg_build_autotune(svg_mesh* m, const svg_build_opts* opts, int32_t max_trials, svg_build_opts* best,
                              double* best_ms);

svg_status svg_graph_stats(const svg_graph* g, svg_build_stats* st);

/* Per-source counters (any pointer may be NULL), n = number of built sources:
 * windows propagated, window-queue high-water mark, flags (bit0 queue drop,
 * bit1 reference-table overflow, bit2 watchdog, bit3 reference-undefined). */
svg_status svg_graph_source_stats(const svg_graph* g, int32_t* windows, int32_t* max_queue, int32_t* flags);

/* SVG::FreeSVGStructure (SVG.cu:149-155). */
void svg_graph_free(svg_graph* g);

/* Kernel form of the query calls on this graph.  CLUSTER (default): one query
 * per thread-block cluster of 8-16 SMs, few queries in flight so that their
 * state stays in L2.  PLAIN: one query per thread block, the reference's
 * one-search-at-a-time form (SVG::SolveSSSD / SolveMSAD, SVG.cu:241-413),
 * kept as the baseline.  Results are the same in both forms. */
enum { SVG_QUERY_CLUSTER = 0, SVG_QUERY_PLAIN = 1 };
svg_status svg_graph_set_query_form(svg_graph* g, int32_t form);

/* Vertex count, edge count, K of the build. */
svg_status svg_graph_counts(const svg_graph* g, int32_t* nv, int64_t* nnz, int32_t* K);

/* SVG::CopySVGToHost (SVG.cu:184-206), as CSR: offsets[nv+1], adj[nnz],
 * dist[nnz] (any may be NULL).  Rows are in ascending adjacent-vertex order,
 * row v holding at most K edges, exactly the reference's d_svg rows. */
svg_status svg_graph_copy_csr(const svg_graph* g, int64_t* offsets, int32_t* adj, double* dist);

/* Full reference-layout rows: tails[nv] and nodes[nnz] (packed CSR order). */
svg_status svg_graph_copy_nodes(const svg_graph* g, int32_t* tails, svg_node* nodes);

/* Device pointers of the resident CSR (for callers that keep data on the GPU). */
svg_status svg_graph_device_csr(const svg_graph* g, const int64_t** offsets, const int32_t** adj,
                                const double** dist);

/* SVG::SaveSVGToFile / LoadSVGFromFile (SVG.cu:208-239): per vertex an int32
 * degree then degree svg_nodes; no header.  Files are interchangeable with
 * the reference's. */
svg_status svg_graph_save(const svg_graph* g, const char* path);
svg_status svg_graph_load(svg_mesh* m, int32_t K, const char* path, svg_graph** out);

/* ---------------------------------------------------------------- queries */

/* SVG::SolveSSSD (SVG.cu:241-251): shortest SVG distance from s[i] to t[i]
 * for n pairs in one batch (DBL_MAX if unreachable).  Host buffers. */
svg_status svg_sssd_batch(svg_graph* g, int32_t n, const int32_t* s, const int32_t* t, double* dist);

/* SVG::SolveMSAD (SVG.cu:354-366): n independent source sets; set q is
 * srcs[set_offsets[q] .. set_offsets[q+1]) with weights (initial distances).
 * dist[q*nv + v] receives the distance of v from set q; src_id (optional)
 * the source whose tree reached v.  A source listed twice keeps the weight
 * of its last occurrence, as the reference does.  Host buffers. */
svg_status svg_msad_batch(svg_graph* g, int32_t n, const int64_t* set_offsets, const int32_t* srcs,
                          const double* weights, double* dist, int32_t* src_id);

/* SVG::SolveMSAD with SVG::GraphDistInfo::pathParentIndex (SVG.cu:396):
 * as svg_msad_batch, plus parent[q*nv + v] = the vertex before v on a
 * shortest path of set q (-1 for a source that kept its own label and for
 * unreached vertices).  Where several predecessors give the same distance,
 * the smallest vertex id is named (the reference names the first its heap
 * relaxes from).  src_id may be NULL.  Host buffers. */
svg_status svg_msad_batch_paths(svg_graph* g, int32_t n, const int64_t* set_offsets, const int32_t* srcs,
                                const double* weights, double* dist, int32_t* src_id, int32_t* parent);

/* SVG::SolveSSSD followed by the reference driver's walk along
 * pathParentIndex from t back to s (kernel.cu:75-82): path[0] = t, ...,
 * path[len-1] = s, path_dist (optional) the distance of each from s; *dist
 * (optional) the s-t distance.  An unreachable t gives len 0 and DBL_MAX.
 * A path longer than cap returns SVG_ERR_ARG with the needed length in *len.
 * Runs a full search from s (device); for many pairs use svg_sssd_batch. */
svg_status svg_sssd_path(svg_graph* g, int32_t s, int32_t t, int32_t cap, int32_t* path, double* path_dist,
                         int32_t* len, double* dist);

/* Same queries on device-resident inputs/outputs (no host copies). */
svg_status svg_sssd_batch_device(svg_graph* g, int32_t n, const int32_t* d_s, const int32_t* d_t,
                                 double* d_dist);
svg_status svg_msad_batch_device(svg_graph* g, int32_t n, const int64_t* d_set_offsets,
                                 const int32_t* d_srcs, const double* d_weights, double* d_dist,
                                 int32_t* d_src_id);

/* Allocation-free build of SVG rows.  No counterpart in the reference (its
 * SVG::Allocation cudaMallocs every buffer); it is for callers that cannot
 * allocate device memory at this point - code whose allocations all belong
 * to an outer framework's pool, or that runs where a cudaMalloc would
 * synchronise the device or break a capture.  The caller provides every
 * buffer; the kernel's scratch is a fixed array inside the library (about
 * 29 MiB per GPU that loads the library, held until the library unloads),
 * with tables sized as svg_build's first pass sizes them at K = 128.
 *   m            a mesh already on the device (svg_mesh_upload, which does
 *                allocate, must have been called earlier)
 *   K            1..128 (queue capacities are the reference's 1023)
 *   [source_begin, source_end)  sources to build, row r = source_begin + r
 *   d_tails      device int32[n]: row length, or a code:
 *                  -1  the source outgrew the fixed tables (svg_build re-runs
 *                      such a source with larger tables);
 *                  -2  an iteration cap stopped the source, or it reached a
 *                      step the reference leaves undefined (svg_build flags
 *                      both in svg_graph_source_stats); the row is not written.
 *                A source where the reference's own fixed hash tables would
 *                overflow gets the same row as svg_build gives it (the exact
 *                ICH's), and is not flagged here.
 *   d_adj, d_dist  device int32[n*K], double[n*K]: padded rows, the same
 *                neighbours and lengths as svg_build's rows
 *   stream       cudaStream_t (NULL: the legacy default stream)
 * Asynchronous: outputs are complete when the stream reaches this point.
 * All calls share the one scratch array, so calls whose kernels could run
 * at the same time on the GPU race; serialise them.  Every call looks up the
 * array's device address on the current device (no allocation); the first
 * call on a device also loads the library's kernels there, so make that
 * first call before any stream capture. */
svg_status svg_build_rows_static(svg_mesh* m, int32_t K, int32_t source_begin, int32_t source_end,
                                 int32_t* d_tails, int32_t* d_adj, double* d_dist, void* stream);

/* ---------------------------------------------------------------- serving
 *
 * A serving loop with no counterpart in the reference (which answers one
 * query at a time on the host, SVG.cu:241-413).  SVGs stay resident on the
 * device; a worker thread batches arriving SSSD and MSAD requests per graph
 * (the oldest pending request plus every other one of the same kind and
 * graph that fits) and launches each batch on one of `lanes` CUDA streams,
 * so batches - and a build running on a builder thread - overlap on the GPU;
 * requests arriving meanwhile join the next batch as soon as a lane frees.
 * Builds are admitted under `hbm_budget`, evicting least-recently-used idle
 * graphs the server built itself; a query for an evicted graph triggers its
 * rebuild and waits for it.  Results are identical to the synchronous batch
 * calls above. */
typedef struct svg_server svg_server;

typedef struct svg_server_opts {
    int64_t hbm_budget;         /* device bytes for resident graphs, query scratch, staging and builds */
    int32_t lanes;              /* concurrent batches (CUDA streams); 0: one per resident query cluster */
    int32_t max_batch;          /* SSSD requests per batch */
    int32_t slots_per_lane;     /* queries of one batch served at once (0: the GPU's share of the lane) */
    int32_t cluster;            /* blocks per query: 0 automatic cluster, -1 one block (plain form), 8 or 16 */
    int64_t staging_in_bytes;   /* per lane: request inputs (pinned host + device) */
    int64_t staging_out_bytes;  /* per lane: results (an MSAD result is 12 bytes per vertex) */
    int32_t max_batch_msad;     /* MSAD requests per batch (each is a whole-graph search) */
    int32_t build_blocks_per_sm;/* build kernel blocks per SM while serving (the rest of each SM stays free
                                   for query blocks); 0: as many as fit (fastest build, queries wait) */
} svg_server_opts;

typedef struct svg_server_result {
    int64_t ticket;
    int32_t status;             /* svg_status of the request */
    int32_t kind;               /* 0 SSSD, 1 MSAD, 2 build */
    int32_t graph_id;
    int32_t n;                  /* MSAD: number of vertices in the result */
    double latency_ms;          /* submit -> result on the host */
    double dist;                /* SSSD distance (DBL_MAX if unreachable) */
    int64_t edges;              /* build: SVG edges */
    double build_ms;            /* build: device time of the build */
} svg_server_result;

typedef struct svg_server_stats_t {
    int64_t pending;
    int64_t batches;
    int64_t batched_requests;
    int64_t resident_bytes;
    int64_t evictions;
    int64_t rebuilds;
    int64_t resident_graphs;
} svg_server_stats_t;

void svg_server_opts_default(svg_server_opts* o);
svg_status svg_server_create(const svg_server_opts* opts, svg_server** out);
void svg_server_free(svg_server* s);
/* Serve an already built graph (owned by the caller, never evicted). */
svg_status svg_server_add_graph(svg_server* s, svg_graph* g, int32_t* graph_id);
/* Build (asynchronously) and serve the SVG of mesh m; graph_id is usable at once. */
svg_status svg_server_submit_build(svg_server* s, svg_mesh* m, const svg_build_opts* opts, int32_t* graph_id,
                                   int64_t* ticket);
svg_status svg_server_submit_sssd(svg_server* s, int32_t graph_id, int32_t src, int32_t dst, int64_t* ticket);
svg_status svg_server_submit_msad(svg_server* s, int32_t graph_id, int32_t n, const int32_t* srcs,
                                  const double* weights, int64_t* ticket);
/* As svg_server_submit_msad, with the result written straight into the
 * caller's host buffers dists[V] and src_ids[V] (either may be NULL to drop
 * it); they must stay valid until the request is finished. */
svg_status svg_server_submit_msad_into(svg_server* s, int32_t graph_id, int32_t n, const int32_t* srcs,
                                       const double* weights, double* dists, int32_t* src_ids, int64_t* ticket);
/* Wait for one request (timeout_s < 0: no limit). */
svg_status svg_server_wait(svg_server* s, int64_t ticket, double timeout_s, svg_server_result* res);
/* Completed requests not yet taken (up to max). */
svg_status svg_server_poll(svg_server* s, int32_t max, svg_server_result* res, int32_t* n);
/* Copy an MSAD result (dists[n], src_ids[n], either may be NULL) and release the request. */
svg_status svg_server_take(svg_server* s, int64_t ticket, double* dists, int32_t* src_ids);
svg_status svg_server_stats(svg_server* s, svg_server_stats_t* st);
/* Ids of the graphs resident now (up to max), most recently used first. */
svg_status svg_server_resident(svg_server* s, int32_t max, int32_t* graph_ids, int32_t* n);

/* Device memory freed by the library (graphs, build scratch, query buffers)
 * is cached for reuse; this returns all cached blocks to CUDA and reports how
 * many bytes it released.  No counterpart in the reference (it cudaMallocs
 * and cudaFrees every buffer). */
size_t svg_trim_device_cache(void);

/* Device bytes the library holds: in use by live objects, the high-water mark
 * of that since the last reset, and cached for reuse.  reset_peak != 0 sets
 * the high-water mark to the current use.  No counterpart in the reference. */
void svg_device_memory(int64_t* in_use, int64_t* peak, int64_t* cached, int32_t reset_peak);

/* Measured FP64 pipe rate of the current GPU: fused multiply-adds per second
 * of a kernel that keeps every SM's FP64 units busy (CUDA events, ~0.1 s).
 * The denominator of the build kernel's FP64 roofline (each of its FP64 adds,
 * multiplies, divides and square roots issues on the same pipe).  No
 * counterpart in the reference. */
svg_status svg_device_fp64_rate(double* fma_per_s);

/* Synchronise the library's stream; returns the device time in ms since the
 * previous svg_timer_mark (CUDA events on the library stream). */
svg_status svg_timer_mark(double* ms_since_last);

#ifdef __cplusplus
}
#endif
#endif
