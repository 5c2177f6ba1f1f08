/* Plain-C restatement of the reference's SVG construction and graph search.
 *
 * TEST ORACLE ONLY: loaded by tests/, the smoke check and bench.py's
 * CPU-baseline leg to check the CUDA product; never linked into it.
 *
 * Pinned against the reference itself (oracle/_ref, the reference's own
 * sources compiled as host C++) and against committed golden fixtures.
 */
#ifndef SVG_ORACLE_H
#define SVG_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same 40-byte layout as SVG::SVGNode (SVG.cuh:21-27). */
typedef struct om_node {
    int32_t adj;
    int32_t pad_;
    double dist;
    uint32_t next_to_src_edge;
    uint32_t next_to_dst_edge;
    double next_to_src_x;
    double next_to_dst_x;
} om_node;

typedef struct om_mesh om_mesh;

/* Half-edge mesh from arrays (Mesh::LoadFromFile, Mesh.cu:62-123), boundary
 * half-edges get twin -1 (the reference leaves 0 there, Mesh.cu:62). */
int om_mesh_create(int nv, const double* pos, int nf, const int32_t* faces, om_mesh** out);
void om_mesh_free(om_mesh* m);
void om_mesh_counts(const om_mesh* m, int* nv, int* nf, int* ne);
void om_mesh_export(const om_mesh* m, int32_t* he_v0, int32_t* he_twin, double* he_len,
                    double* angle, int32_t* first_edge);

/* SVG rows for `nsrc` sources (constructSVG body, SVG.cu:34-76).
 * nodes: nsrc*K slots, row r holds tails[r] nodes.  stats: nsrc*5 ints
 * {windows generated, max window queue, max pseudo queue, vertices counted,
 * flags} or NULL.  flags bit0: a hash table overflowed into its sink slot;
 * bit1: the watchdog cap on loop iterations was hit.  Returns seconds. */
double om_build(const om_mesh* m, int K, unsigned split_coef, unsigned vert_coef, int win_cap,
                int pseudo_cap, const int32_t* sources, int nsrc, int nthreads, int32_t* tails,
                om_node* nodes, int32_t* stats);

/* Per-vertex ICH distances (K-limited, or K=-1 exhaustive) with explicit
 * table sizes and queue capacities.  dist: nsrc*V. */
double om_ich_distances(const om_mesh* m, int K, unsigned split_size, unsigned vert_size,
                        int win_cap, int pseudo_cap, const int32_t* sources, int nsrc,
                        int nthreads, double* dist, int32_t* stats);

/* Graph search on a CSR graph (offsets[V+1], adj, w): A* with the Euclidean
 * heuristic for (s,t) pairs (SVG::SolveSSSD, SVG.cu:241-251 + Astar 369-413)
 * and multi-source Dijkstra (SVG::SolveMSAD, SVG.cu:354-366). */
double om_sssd(const om_mesh* m, const int64_t* offsets, const int32_t* adj, const double* w,
               int n, const int32_t* s, const int32_t* t, double* dist_out);
double om_msad(const om_mesh* m, const int64_t* offsets, const int32_t* adj, const double* w,
               int ns, const int32_t* srcs, const double* weights, double* dist_out,
               int32_t* src_out);

#ifdef __cplusplus
}
#endif
#endif
