/* oracle/orc_grid.h -- exact CPU neighbour search for the oracle.
 *
 * TEST INFRASTRUCTURE ONLY (see gizmo_oracle.h).
 *
 * A Morton-ordered octree pyramid over a periodic box: particles are
 * counting-sorted into 8^F fine cells by their interleaved cell key, so every
 * octree node at every level owns one contiguous run of the sorted order
 * (prefix[] gives its bounds) and carries the largest kernel length of its
 * members. A query descends the pyramid, pruning nodes whose periodic
 * minimum distance is beyond reach (h_i for one-way, max(h_i, node h max)
 * for symmetric), and tests the survivors with the reference predicates:
 *   one-way   : r2 < h_i^2                         (density_loop.h:1163-1171)
 *   symmetric : !(r2 >= h_i^2 && r2 >= h_j^2)      (hydro_functions.h:77-83,
 *               gradient_functions.h:351)
 * where r2 is the squared periodic minimum-image separation computed exactly
 * as the reference does (NEAREST_XYZ, declarations/macros.h:58-109).
 */
#ifndef ORC_GRID_H
#define ORC_GRID_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_grid {
    int       F;          /* fine level: 2^F cells per axis */
    int       n;
    double    box;
    int      *order;      /* [n] particle index by sorted position */
    int64_t  *prefix;     /* [8^F + 1] first sorted position of each fine cell */
    double   *hmax;       /* pyramid of node h maxima, level offsets below */
    int64_t   level_off[12];
} orc_grid;

int  orc_grid_build(orc_grid *g, const double *pos, const double *h, int n, double box);
void orc_grid_free(orc_grid *g);

/* Minimum-image separation, reference operation order. */
static inline double orc_wrap(double x, double box, double half)
{
    return (x > half) ? (x - box) : ((x < -half) ? (x + box) : x);
}

/* Collects candidate particles (indices into the original arrays) for a
 * query at x with one-way reach hi (symmetric != 0 widens reach by the
 * node h maxima). Returns the count; cand must hold n entries worst case,
 * *cap is its size (grown with realloc when needed). */
int orc_grid_candidates(const orc_grid *g, const double *x, double hi, int symmetric,
                        int **cand, int *cap);

#ifdef __cplusplus
}
#endif
#endif
