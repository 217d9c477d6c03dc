/* oracle/orc_grid.c -- exact CPU neighbour search (see orc_grid.h).
 * TEST INFRASTRUCTURE ONLY. */
#include "orc_grid.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static uint32_t spread3(uint32_t x)
{
    x &= 0x3ff;
    x = (x | (x << 16)) & 0x030000ff;
    x = (x | (x << 8)) & 0x0300f00f;
    x = (x | (x << 4)) & 0x030c30c3;
    x = (x | (x << 2)) & 0x09249249;
    return x;
}

static uint32_t compact3(uint32_t x)
{
    x &= 0x09249249;
    x = (x | (x >> 2)) & 0x030c30c3;
    x = (x | (x >> 4)) & 0x0300f00f;
    x = (x | (x >> 8)) & 0x030000ff;
    x = (x | (x >> 16)) & 0x000003ff;
    return x;
}

static inline uint32_t morton3(uint32_t a, uint32_t b, uint32_t c)
{
    return spread3(a) | (spread3(b) << 1) | (spread3(c) << 2);
}

static inline int cell_of(double x, double box, int G)
{
    int c = (int)(x / box * (double)G);
    if (c < 0) c = 0;
    if (c >= G) c = G - 1;
    return c;
}

int orc_grid_build(orc_grid *g, const double *pos, const double *h, int n, double box)
{
    memset(g, 0, sizeof(*g));
    int F = 1;
    while (F < 8 && ((int64_t)1 << (3 * F)) < (int64_t)n) F++;
    const int G = 1 << F;
    const int64_t C = (int64_t)1 << (3 * F);
    g->F = F;
    g->n = n;
    g->box = box;
    g->order = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    g->prefix = (int64_t *)calloc((size_t)(C + 1), sizeof(int64_t));
    uint32_t *key = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(n > 0 ? n : 1));
    if (!g->order || !g->prefix || !key) { free(key); orc_grid_free(g); return 1; }
    for (int i = 0; i < n; i++) {
        key[i] = morton3((uint32_t)cell_of(pos[3 * i + 0], box, G), (uint32_t)cell_of(pos[3 * i + 1], box, G),
                         (uint32_t)cell_of(pos[3 * i + 2], box, G));
        g->prefix[key[i] + 1]++;
    }
    for (int64_t c = 0; c < C; c++) g->prefix[c + 1] += g->prefix[c];
    int64_t *fill = (int64_t *)malloc(sizeof(int64_t) * (size_t)C);
    memcpy(fill, g->prefix, sizeof(int64_t) * (size_t)C);
    for (int i = 0; i < n; i++) g->order[fill[key[i]]++] = i; /* stable: ascending index within a cell */
    free(fill);
    /* node h maxima, fine level first */
    int64_t total = 0;
    for (int L = 0; L <= F; L++) { g->level_off[L] = total; total += (int64_t)1 << (3 * L); }
    g->hmax = (double *)calloc((size_t)total, sizeof(double));
    double *fine = g->hmax + g->level_off[F];
    for (int i = 0; i < n; i++) {
        double hv = h ? h[i] : 0.0;
        if (hv > fine[key[i]]) fine[key[i]] = hv;
    }
    for (int L = F - 1; L >= 0; L--) {
        double *lv = g->hmax + g->level_off[L];
        const double *ch = g->hmax + g->level_off[L + 1];
        const int64_t nn = (int64_t)1 << (3 * L);
        for (int64_t m = 0; m < nn; m++) {
            double v = 0;
            for (int k = 0; k < 8; k++) if (ch[8 * m + k] > v) v = ch[8 * m + k];
            lv[m] = v;
        }
    }
    free(key);
    return 0;
}

void orc_grid_free(orc_grid *g)
{
    free(g->order);
    free(g->prefix);
    free(g->hmax);
    memset(g, 0, sizeof(*g));
}

/* periodic distance from x to the interval [lo, lo+s) along one axis */
static inline double axis_gap(double x, double lo, double s, double box)
{
    double c = lo + 0.5 * s;
    double d = fabs(x - c);
    if (d > 0.5 * box) d = box - d;
    d -= 0.5 * s;
    return d > 0 ? d : 0;
}

static int push_range(int **cand, int *cap, int cnt, const orc_grid *g, int64_t a, int64_t b)
{
    int64_t need = cnt + (b - a);
    if (need > *cap) {
        int nc = *cap > 0 ? *cap : 256;
        while (nc < need) nc *= 2;
        int *p = (int *)realloc(*cand, sizeof(int) * (size_t)nc);
        if (!p) return -1;
        *cand = p;
        *cap = nc;
    }
    for (int64_t k = a; k < b; k++) (*cand)[cnt++] = g->order[k];
    return cnt;
}

int orc_grid_candidates(const orc_grid *g, const double *x, double hi, int symmetric, int **cand, int *cap)
{
    int cnt = 0;
    int stackL[8 * 12 + 8];
    int64_t stackM[8 * 12 + 8];
    int sp = 0;
    stackL[sp] = 0;
    stackM[sp] = 0;
    sp++;
    const int F = g->F;
    while (sp > 0) {
        sp--;
        const int L = stackL[sp];
        const int64_t m = stackM[sp];
        const int sh = 3 * (F - L);
        const int64_t a = g->prefix[m << sh], b = g->prefix[(m + 1) << sh];
        if (a == b) continue;
        double reach = hi;
        if (symmetric) {
            double hn = g->hmax[g->level_off[L] + m];
            if (hn > reach) reach = hn;
        }
        const double s = g->box / (double)(1 << L);
        const double ax = (double)compact3((uint32_t)m) * s;
        const double ay = (double)compact3((uint32_t)(m >> 1)) * s;
        const double az = (double)compact3((uint32_t)(m >> 2)) * s;
        const double gx = axis_gap(x[0], ax, s, g->box), gy = axis_gap(x[1], ay, s, g->box),
                     gz = axis_gap(x[2], az, s, g->box);
        const double d2 = gx * gx + gy * gy + gz * gz;
        /* conservative prune: a node is dropped only when clearly out of reach */
        if (d2 > reach * reach * (1.0 + 1e-9) + 1e-300) continue;
        if (L == F || (b - a) <= 32) {
            cnt = push_range(cand, cap, cnt, g, a, b);
            if (cnt < 0) return -1;
        } else {
            for (int k = 7; k >= 0; k--) {
                stackL[sp] = L + 1;
                stackM[sp] = 8 * m + k;
                sp++;
            }
        }
    }
    return cnt;
}
