/*
 * cgb200 synthetic-graph generators.  The reference has no generator (its
 * only synthetic step is txtToBin's rand()%99+1 edge weights,
 * Basic/Graph/txtToBin.hpp:74); these build the seeded inputs the engine is
 * measured on straight into HBM, in the CSR format of load_binFile
 * (Basic/Other/IO.hpp:44-92): sorted, duplicate-free, self-loop-free lists.
 * Every value is a pure function of the seed (counter-based splitmix64), so
 * the CPU twin in the test oracle rebuilds the same graph bit for bit.
 */
#ifndef CGB200_GEN_H
#define CGB200_GEN_H

#include "cgb200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* RMAT: edge_factor * 2^scale edges drawn with quadrant probabilities a, b,
 * c (d = 1 - a - b - c), ids optionally scrambled by a seeded bijection,
 * self-loops and duplicates removed, optionally symmetrised.  wmax > 0 gives
 * weights uniform in [1, wmax] (equal in both directions when symmetrised);
 * wmax = 0 gives no weight array. */
cgb_status cgb_gen_rmat(uint32_t scale, uint32_t edge_factor, uint64_t seed, double a, double b, double c,
                        int scramble, int symmetrise, uint32_t wmax, int device, cgb_graph** out);

/* Chung-Lu power-law graph: `draws` edges whose endpoints are both drawn
 * with probability proportional to a vertex weight floor(2^40 / (i + i0))
 * (rank-i expected degree ~ 1 / (i + i0): degree-distribution exponent 2,
 * largest expected degree set by weight_offset = i0), out- and in-ranks
 * spread over the ids by two seeded affine permutations; self-loops and
 * duplicates removed, optionally symmetrised, weights as for RMAT. */
cgb_status cgb_gen_chunglu(uint32_t vertices, uint64_t draws, uint32_t weight_offset, uint64_t seed, int symmetrise,
                           uint32_t wmax, int device, cgb_graph** out);
/* rows x cols 4-neighbour grid (undirected), weights uniform in [1, wmax]. */
cgb_status cgb_gen_grid(uint32_t rows, uint32_t cols, uint64_t seed, uint32_t wmax, int device, cgb_graph** out);

/* Copies the resident CSR to caller buffers (host or device): offsets V+1,
 * dest E, weight E (may be NULL; ignored when the graph has no weights). */
cgb_status cgb_graph_download(const cgb_graph* g, uint32_t* offsets, uint32_t* dest, uint32_t* weight);

#ifdef __cplusplus
}
#endif
#endif /* CGB200_GEN_H */
