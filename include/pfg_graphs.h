/*
 * pfg_graphs.h - host-side graph substrate of libpfg_b200.so: weight-sorted
 * CSR construction, seeded synthetic generators for the benchmark workloads,
 * and loaders for real road networks.
 *
 * The CSR contract is the reference's (include/graph.h:31-48,
 * src/graph.cpp:23-104): self loops dropped, weights clamped to >= 1, rows
 * grouped by source with a counting sort and each row sorted by (w, dst), so
 * the light arcs (w <= Delta) of a row are a prefix. hScale is the largest
 * admissible heuristic scale min(w / |p(u) - p(v)|) over arcs with a
 * positive length.
 *
 * Randomness is SplitMix64 seeded as in the reference's Rng
 * (include/common.h:44-56): state = seed * 0x9E3779B97F4A7C15 + 0x1234567.
 */
#ifndef PFG_GRAPHS_H_
#define PFG_GRAPHS_H_

#include <stdint.h>
#include "pfg.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pfg_graph pfg_graph;

/* Mirrors the statistics of CSRGraph (reference: include/graph.h:31-48). */
typedef struct pfg_graph_info {
    uint32_t n, m;
    uint32_t min_w, max_w, max_deg;
    int32_t has_xy;
    double avg_w, avg_deg, h_scale;
} pfg_graph_info;

/* Builds a CSR from an arc list (reference: buildCSR, src/graph.cpp:23-104).
 * x, y: optional coordinates (both NULL or both length n). */
PFG_API pfg_status pfg_graph_from_edges(uint32_t n, uint64_t m_in, const uint32_t* src,
                                const uint32_t* dst, const uint32_t* w, const double* x,
                                const double* y, pfg_graph** out);

/* The same CSR built on the GPU (self loops dropped, w < 1 raised to 1, rows
 * sorted by (w, dst), statistics and h_scale): a result identical word for
 * word to pfg_graph_from_edges, for arc lists too large to sort on the host
 * quickly (extension; replaces the host counting sort and per-row sort of
 * buildCSR, src/graph.cpp:23-104). Host arrays in, host graph out. */
PFG_API pfg_status pfg_graph_from_edges_gpu(uint32_t n, uint64_t m_in, const uint32_t* src,
                                    const uint32_t* dst, const uint32_t* w, const double* x,
                                    const double* y, int32_t device, pfg_graph** out);

/* The device part of pfg_graph_from_edges_gpu for arcs already on the GPU:
 * d_src / d_dst / d_w [m_in], optional d_x / d_y [n]; writes d_row [n+1],
 * d_col and d_w_out (the first info->m entries, at most m_in) and the
 * statistics into *info. Allocates its scratch with cudaMalloc; returns after
 * the work on `stream` (a cudaStream_t, NULL = default stream) is done. */
PFG_API pfg_status pfg_csr_build_device(uint32_t n, uint64_t m_in, const uint32_t* d_src,
                                const uint32_t* d_dst, const uint32_t* d_w, const double* d_x,
                                const double* d_y, uint32_t* d_row, uint32_t* d_col,
                                uint32_t* d_w_out, pfg_graph_info* info, int32_t device,
                                void* stream);

/* rows x cols grid at integer coordinates (x = column, y = row), arcs both ways
 * to the 4 neighbours, each arc its own weight llround(100 * U[1.0, 1.5)). */
PFG_API pfg_status pfg_graph_gen_grid(uint32_t rows, uint32_t cols, uint64_t seed, pfg_graph** out);

/* Directed R-MAT: 2^scale vertices, edge_factor * 2^scale samples, quadrant
 * probabilities (a, b, c, 1-a-b-c), self loops dropped, duplicate arcs keep
 * the smallest weight, weights uniform in [w_lo, w_hi]. No coordinates. */
PFG_API pfg_status pfg_graph_gen_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c,
                              uint32_t w_lo, uint32_t w_hi, uint64_t seed, pfg_graph** out);

/* Road-like side x side grid: the 4-neighbour grid above with a fraction
 * `removal` of undirected neighbour pairs deleted, plus a bidirectional
 * shortcut from a fraction `shortcut` of vertices to a uniform vertex within
 * Chebyshev radius `radius`, weight ceil(factor * 100 * Euclidean length). */
PFG_API pfg_status pfg_graph_gen_road(uint32_t side, double removal, double shortcut, uint32_t radius,
                              double factor, uint64_t seed, pfg_graph** out);

/* Disjoint union of graphs: vertex ids of graph i are shifted by the number
 * of vertices before it; coordinates are kept when every input has them. */
PFG_API pfg_status pfg_graph_union(const pfg_graph* const* parts, uint32_t count, pfg_graph** out);

/* DIMACS 9th challenge shortest-path files (.gr arcs "a u v w", 1-based; .co
 * coordinates "v id x y", optional) (reference: loadDIMACS,
 * src/graph.cpp:227-282). co_path may be NULL. */
PFG_API pfg_status pfg_graph_load_dimacs(const char* gr_path, const char* co_path, pfg_graph** out);
/* SNAP edge list "u v [w]" with '#'/'%' comments; missing weights are
 * 1 + hash(min,max) % max_w; symmetrize adds the reverse arc (reference:
 * loadSNAP, src/graph.cpp:284-316). */
PFG_API pfg_status pfg_graph_load_snap(const char* path, int32_t symmetrize, uint32_t max_w,
                               uint64_t seed, pfg_graph** out);
/* Binary cache in the reference's PFCSR001 layout (src/graph.cpp:320-367). */
PFG_API pfg_status pfg_graph_save_binary(const pfg_graph* g, const char* path);
PFG_API pfg_status pfg_graph_load_binary(const char* path, pfg_graph** out);

PFG_API pfg_status pfg_graph_get_info(const pfg_graph* g, pfg_graph_info* out);
PFG_API const uint32_t* pfg_graph_row_offsets(const pfg_graph* g);
PFG_API const uint32_t* pfg_graph_col_indices(const pfg_graph* g);
PFG_API const uint32_t* pfg_graph_weights(const pfg_graph* g);
PFG_API const double* pfg_graph_x(const pfg_graph* g); /* NULL without coordinates */
PFG_API const double* pfg_graph_y(const pfg_graph* g);
PFG_API void pfg_graph_free(pfg_graph* g);

/* k vertices with out-degree > 0, drawn with Rng(seed).below(n) (reference:
 * pickSources, src/graph.cpp:369-378). */
PFG_API pfg_status pfg_graph_pick_sources(const pfg_graph* g, uint32_t count, uint64_t seed,
                                  uint32_t* out);

#ifdef __cplusplus
}
#endif
#endif /* PFG_GRAPHS_H_ */
