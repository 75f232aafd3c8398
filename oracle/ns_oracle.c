/* ns_oracle.c -- CPU restatement of the reference's random neighbourhood
 * moves (TEST INFRASTRUCTURE ONLY; only tests/ load it):
 *
 *   glibc random()/srandom() (TYPE_3: degree 31, separation 3), the generator
 *   NeighbourSearch draws from (neighbourSearch.cpp:29-32,431-446);
 *   NeighbourSearch::reset_ant / search / exchange / exchange_1 / insertion /
 *   insertion_1 / inversion (neighbourSearch.cpp:40-427) and Move::apply
 *   (move.cpp:17-80).
 *
 * The reference's rejection loops ("while (sz <= 3)", "while (n1 == 0)") spin
 * forever when no route qualifies; here each gives up after a bounded number
 * of draws and the proposal is "none".  Float expressions keep the reference's
 * evaluation order (built with -ffp-contract=off). */
#include "aco_oracle.h"

#include <stdint.h>
#include <stdlib.h>

#define EPS_F 0.001f /* utilities.h:19 */

void orc_srandom(orc_rng *g, unsigned seed)
{
    int32_t word = (int32_t)(seed ? seed : 1u);
    g->r[0] = (uint32_t)word;
    for (int i = 1; i < 31; i++) {
        const long hi = word / 127773, lo = word % 127773;
        long w = 16807 * lo - 2836 * hi;
        if (w < 0) w += 2147483647;
        word = (int32_t)w;
        g->r[i] = (uint32_t)word;
    }
    g->f = 3;
    g->b = 0;
    for (int k = 0; k < 310; k++) (void)orc_random(g);
}

int32_t orc_random(orc_rng *g)
{
    const uint32_t v = g->r[g->f] += g->r[g->b];
    if (++g->f >= 31) g->f = 0;
    if (++g->b >= 31) g->b = 0;
    return (int32_t)(v >> 1);
}

typedef struct { int beg, end, load; float dist; } route_t;

static int reset_routes(int n, const float *dist, const int *demand, const int *tour, int size, route_t *rt)
{
    int k = 0, beg = 0, load = 0;
    float d = 0.f;
    for (int i = 1; i < size; i++) {
        load += demand[tour[i]];
        d += dist[(size_t)tour[i - 1] * n + tour[i]];
        if (tour[i] == 0) {
            rt[k].beg = beg; rt[k].end = i; rt[k].load = load; rt[k].dist = d;
            k++;
            beg = i; load = 0; d = 0.f;
        }
    }
    return k;
}

#define D(a, b) dist[(size_t)(a) * n + (b)]
#define TRIES 4096

static int rnd_route(orc_rng *g, int nr) { return (int)orc_random(g) % nr; }
static int rnd_pos(orc_rng *g, const route_t *r) { return r->beg + orc_random(g) % (r->end - r->beg); }

/* a route with at least two customers, or -1 */
static int big_route(orc_rng *g, const route_t *rt, int nr)
{
    for (int t = 0; t < TRIES; t++) {
        const int r = rnd_route(g, nr);
        if (rt[r].end - rt[r].beg + 1 > 3) return r;
    }
    return -1;
}

static int customer_pos(orc_rng *g, const route_t *r, int avoid)
{
    for (int t = 0; t < TRIES; t++) {
        const int p = rnd_pos(g, r);
        if (p != r->beg && p != avoid) return p;
    }
    return -1;
}

static void none(orc_move *m) { m->type = -1; m->valid = 0; m->gain = 0.f; m->pos1 = m->pos2 = 0; }

static void exchange_1(int n, const float *dist, float max_dist, float serv, const int *tour, const route_t *rt,
                       int nr, orc_rng *g, orc_move *m)
{
    const int r = big_route(g, rt, nr);
    if (r < 0) { none(m); return; }
    const route_t *ro = &rt[r];
    int p1 = customer_pos(g, ro, -1);
    int p2 = p1 < 0 ? -1 : customer_pos(g, ro, p1);
    if (p2 < 0) { none(m); return; }
    if (p1 > p2) { const int t = p1; p1 = p2; p2 = t; }
    const int n1 = tour[p1], n2 = tour[p2];
    const int p_n1 = tour[p1 - 1], p_n2 = tour[p2 - 1], s_n1 = tour[p1 + 1], s_n2 = tour[p2 + 1];
    float gain;
    if (p2 - p1 == 1)
        gain = -(D(p_n1, n1) + D(n2, s_n2)) + (D(p_n1, n2) + D(n1, s_n2));
    else
        gain = -(D(p_n1, n1) + D(n1, s_n1) + D(p_n2, n2) + D(n2, s_n2)) +
               (D(p_n1, n2) + D(n2, s_n1) + D(p_n2, n1) + D(n1, s_n2));
    const float d = ro->dist + (ro->end - ro->beg - 1) * serv + gain;
    m->type = 0; m->valid = !(d > max_dist); m->gain = gain; m->pos1 = p1; m->pos2 = p2;
}

static void exchange(int n, const float *dist, const int *demand, int cap, float max_dist, float serv,
                     const int *tour, const route_t *rt, int nr, orc_rng *g, orc_move *m)
{
    const int r1 = rnd_route(g, nr), r2 = rnd_route(g, nr);
    if (r1 == r2) { exchange_1(n, dist, max_dist, serv, tour, rt, nr, g, m); return; }
    int p1 = -1, p2 = -1, n1 = 0, n2 = 0;
    for (int t = 0; t < TRIES && n1 == 0; t++) { p1 = rnd_pos(g, &rt[r1]); n1 = tour[p1]; }
    for (int t = 0; t < TRIES && n2 == 0; t++) { p2 = rnd_pos(g, &rt[r2]); n2 = tour[p2]; }
    if (n1 == 0 || n2 == 0) { none(m); return; }
    const int p_n1 = tour[p1 - 1], p_n2 = tour[p2 - 1], s_n1 = tour[p1 + 1], s_n2 = tour[p2 + 1];
    const float gain = -(D(p_n1, n1) + D(n1, s_n1) + D(p_n2, n2) + D(n2, s_n2)) +
                       (D(p_n1, n2) + D(n2, s_n1) + D(p_n2, n1) + D(n1, s_n2));
    const float d1 = rt[r1].dist + (rt[r1].end - rt[r1].beg - 1) * serv - (D(p_n1, n1) + D(n1, s_n1)) +
                     (D(p_n1, n2) + D(n2, s_n1));
    const float d2 = rt[r2].dist + (rt[r2].end - rt[r2].beg - 1) * serv - (D(p_n2, n2) + D(n2, s_n2)) +
                     (D(p_n2, n1) + D(n1, s_n2));
    const int l1 = rt[r1].load - demand[n1] + demand[n2], l2 = rt[r2].load - demand[n2] + demand[n1];
    m->type = 0;
    m->valid = !((l1 > cap || l2 > cap) || (d1 > max_dist || d2 > max_dist));
    m->gain = gain; m->pos1 = p1; m->pos2 = p2;
}

static float insertion_gain(int n, const float *dist, const int *tour, int p1, int p2)
{
    const int n1 = tour[p1], n2 = tour[p2];
    const int p_n1 = tour[p1 - 1], p_n2 = tour[p2 - 1], s_n1 = tour[p1 + 1], s_n2 = tour[p2 + 1];
    if (p1 > p2)
        return -(D(p_n1, n1) + D(n1, s_n1) + D(p_n2, n2)) + (D(n1, n2) + D(p_n2, n1) + D(p_n1, s_n1));
    return -(D(p_n1, n1) + D(n1, s_n1) + D(n2, s_n2)) + (D(n2, n1) + D(n1, s_n2) + D(p_n1, s_n1));
}

static void insertion_1(int n, const float *dist, float max_dist, float serv, const int *tour, const route_t *rt,
                        int nr, orc_rng *g, orc_move *m)
{
    const int r = big_route(g, rt, nr);
    if (r < 0) { none(m); return; }
    const route_t *ro = &rt[r];
    const int p1 = customer_pos(g, ro, -1);
    const int p2 = p1 < 0 ? -1 : customer_pos(g, ro, p1);
    if (p2 < 0) { none(m); return; }
    const float gain = insertion_gain(n, dist, tour, p1, p2);
    const float d = ro->dist + (ro->end - ro->beg - 1) * serv + gain;
    m->type = 1; m->valid = !(d > max_dist); m->gain = gain; m->pos1 = p1; m->pos2 = p2;
}

static void insertion(int n, const float *dist, const int *demand, int cap, float max_dist, float serv,
                      const int *tour, const route_t *rt, int nr, orc_rng *g, orc_move *m)
{
    const int r1 = big_route(g, rt, nr);
    if (r1 < 0) { none(m); return; }
    const int r2 = rnd_route(g, nr);
    if (r1 == r2) { insertion_1(n, dist, max_dist, serv, tour, rt, nr, g, m); return; }
    const int p1 = customer_pos(g, &rt[r1], -1), p2 = customer_pos(g, &rt[r2], -1);
    if (p1 < 0 || p2 < 0) { none(m); return; }
    const int n1 = tour[p1], n2 = tour[p2];
    const int p_n2 = tour[p2 - 1], s_n2 = tour[p2 + 1];
    const float gain = insertion_gain(n, dist, tour, p1, p2);
    const route_t *q = &rt[r2];
    float d2;
    if (p1 > p2)
        d2 = q->dist + (q->end - q->beg) * serv - (D(p_n2, n2)) + (D(n1, n2) + D(p_n2, n1));
    else
        d2 = q->dist + (q->end - q->beg) * serv - (D(n2, s_n2)) + (D(n2, n1) + D(n1, s_n2));
    const int l2 = q->load + demand[n1];
    m->type = 1; m->valid = !(l2 > cap || d2 > max_dist); m->gain = gain; m->pos1 = p1; m->pos2 = p2;
}

static void inversion(int n, const float *dist, float max_dist, float serv, const int *tour, const route_t *rt,
                      int nr, orc_rng *g, orc_move *m)
{
    const int r = big_route(g, rt, nr);
    if (r < 0) { none(m); return; }
    const route_t *ro = &rt[r];
    int p1 = customer_pos(g, ro, -1);
    int p2 = p1 < 0 ? -1 : customer_pos(g, ro, p1);
    if (p2 < 0) { none(m); return; }
    if (p1 > p2) { const int t = p1; p1 = p2; p2 = t; }
    if (p2 == ro->end - 1 && p1 == ro->beg + 1) { none(m); return; } /* the whole route: no move */
    const int n1 = tour[p1], n2 = tour[p2], p_n1 = tour[p1 - 1], s_n2 = tour[p2 + 1];
    const float gain = -(D(p_n1, n1) + D(n2, s_n2)) + (D(p_n1, n2) + D(n1, s_n2));
    const float d = ro->dist + (ro->end - ro->beg - 1) * serv + gain;
    m->type = 2; m->valid = !(d > max_dist); m->gain = gain; m->pos1 = p1; m->pos2 = p2;
}

void orc_ns_propose(int n, const float *dist, const int *demand, int cap, float max_dist, float serv,
                    const int *tour, int size, orc_rng *g, orc_move *m)
{
    route_t *rt = (route_t *)malloc(sizeof(route_t) * (size_t)(size > 1 ? size : 1));
    const int nr = reset_routes(n, dist, demand, tour, size, rt);
    if (nr < 1) { none(m); free(rt); return; }
    switch (orc_random(g) % 3) {
    case 0: exchange(n, dist, demand, cap, max_dist, serv, tour, rt, nr, g, m); break;
    case 1: insertion(n, dist, demand, cap, max_dist, serv, tour, rt, nr, g, m); break;
    default: inversion(n, dist, max_dist, serv, tour, rt, nr, g, m); break;
    }
    free(rt);
}

void orc_ns_apply(int *tour, const orc_move *m)
{
    int p1 = m->pos1, p2 = m->pos2;
    if (m->type == 0) {
        const int t = tour[p1]; tour[p1] = tour[p2]; tour[p2] = t;
    } else if (m->type == 1) {
        const int t = tour[p1];
        if (p1 < p2) for (int i = p1; i < p2; i++) tour[i] = tour[i + 1];
        else for (int i = p1; i > p2; i--) tour[i] = tour[i - 1];
        tour[p2] = t;
    } else if (m->type == 2) {
        if (p1 > p2) { const int t = p1; p1 = p2; p2 = t; }
        while (p1 < p2) { const int t = tour[p1]; tour[p1] = tour[p2]; tour[p2] = t; p1++; p2--; }
    }
}

unsigned orc_ns_seed(int rnd_seed, int iteration, int ant)
{
    unsigned s = (unsigned)rnd_seed * 2654435761u + (unsigned)iteration * 40503u + (unsigned)ant * 2246822519u;
    s &= 0x7fffffffu;
    return s ? s : 1u;
}

int orc_ns_descent(int n, const float *dist, const int *demand, int cap, float max_dist, float serv, int *tour,
                   int size, unsigned seed, int rounds)
{
    orc_rng g;
    orc_srandom(&g, seed);
    int applied = 0;
    for (int k = 0; k < rounds; k++) {
        orc_move m;
        orc_ns_propose(n, dist, demand, cap, max_dist, serv, tour, size, &g, &m);
        if (m.type >= 0 && m.valid && m.gain < -EPS_F) {
            orc_ns_apply(tour, &m);
            applied++;
        }
    }
    return applied;
}
#undef D
