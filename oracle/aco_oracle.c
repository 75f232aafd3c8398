/*
 * aco_oracle.c -- CPU restatement of the reference's CVRP ACO iteration.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker the CUDA path is compared
 * against; it is never linked into the product library.  Only tests/, the
 * package smoke check and bench.py's cpu_baseline / --impl reference legs load it.
 *
 * Reference: i-sunny/cvrp_aco_ocl.  The reference's hot path is OpenCL C
 * (cvrp_ocl/gpu/kernel.cl) driven by cvrp_ocl/gpu/g_aco.cpp; it has no CPU ACO.
 * Each function below restates one kernel or host routine and cites it.  The
 * OpenCL work-group of `nloc` work-items is emulated lane by lane: every lane
 * owns its own Park-Miller state and the barrier-separated phases run one after
 * another, which is exact because the phases have no intra-phase races
 * (kernel.cl:331-366).
 *
 * Pinning: tests compare this restatement with the reference's own kernel.cl and
 * g_aco.cpp compiled for the CPU against a fake OpenCL runtime (oracle/refshim),
 * and with the committed golden fixtures under tests/golden/.
 *
 * Floating point: built with -ffp-contract=off; all arithmetic is fp32 in the
 * order the reference writes it.  For integer alpha/beta, pow(x, k) is the exact
 * left-to-right product x*x*...*x (the reference's OpenCL pow has an
 * implementation-defined error of up to 16 ulp, so this rule defines the bits).
 */
#include "aco_oracle.h"

#include <limits.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>

#define IA 16807
#define IM 2147483647
#define IQ 127773
#define IR 2836
#define EPSILON 0.001f /* cvrp_ocl/utilities.h:19, kernel.cl:6 */

/* ran01: Park-Miller minimal standard via Schrage (utilities.cpp:271-288 ==
 * kernel.cl:42-52).  AM = 1.0f/IM is exactly 2^-31 in fp32. */
float orc_ran01(int *idum)
{
    int k = (*idum) / IQ;
    *idum = IA * (*idum - k * IQ) - IR * k;
    if (*idum < 0) *idum += IM;
    return (1.0f / IM) * (float)(*idum);
}

/* (int) of a float the way x86 cvttss2si does it: NaN and out-of-range values
 * become INT_MIN.  The reference's seed formula relies on this conversion when
 * (A-1)*A*A + time overflows int (g_aco.cpp:718). */
int orc_f2i_x86(float v)
{
    if (v != v || v >= 2147483648.0f || v <= -2147483648.0f) return INT_MIN;
    return (int)v;
}

/* Seed generation, g_aco.cpp:714-722:
 *   seed[i] = (int)time(NULL) + (i%A) * ((i%A) + ran01(&rnd_seed)) * A
 * evaluated in fp32 left to right; time(NULL) is replaced by seed_time. */
void orc_make_seeds(int seed_time, int *rnd_seed, int n_ants, int nloc, int *seeds)
{
    int total = n_ants * nloc;
    for (int i = 0; i < total; i++) {
        int m = i % n_ants;
        float r = orc_ran01(rnd_seed);
        float inner = (float)m + r;
        float prod = (float)m * inner;
        prod = prod * (float)n_ants;
        float v = (float)seed_time + prod;
        seeds[i] = orc_f2i_x86(v);
    }
}

/* ---------------------------------------------------------------------- */
/* Distances (vrpHelper.cpp:35-184).                                       */
/* ---------------------------------------------------------------------- */
static float dtrunc_(float x) { int k = (int)x; return (float)k; }

static float dist_euc(const float *x, const float *y, int i, int j)
{ /* round_distance, vrpHelper.cpp:67-81 (no rounding despite the name) */
    float xd = x[i] - x[j];
    float yd = y[i] - y[j];
    return sqrtf(xd * xd + yd * yd);
}

static int dist_ceil(const float *x, const float *y, int i, int j)
{ /* vrpHelper.cpp:83-97 */
    float xd = x[i] - x[j];
    float yd = y[i] - y[j];
    float r = sqrtf(xd * xd + yd * yd);
    return (int)(ceilf(r));
}

static int dist_geo(const float *x, const float *y, int i, int j)
{ /* vrpHelper.cpp:99-136, same mix of float variables and double arithmetic */
    const double PI = 3.14159265358979323846264;
    float deg, min, lati, latj, longi, longj, q1, q2, q3;
    float x1 = x[i], x2 = x[j], y1 = y[i], y2 = y[j];
    deg = dtrunc_(x1); min = x1 - deg; lati = PI * (deg + 5.0 * min / 3.0) / 180.0;
    deg = dtrunc_(x2); min = x2 - deg; latj = PI * (deg + 5.0 * min / 3.0) / 180.0;
    deg = dtrunc_(y1); min = y1 - deg; longi = PI * (deg + 5.0 * min / 3.0) / 180.0;
    deg = dtrunc_(y2); min = y2 - deg; longj = PI * (deg + 5.0 * min / 3.0) / 180.0;
    q1 = cosf(longi - longj); /* float argument: the C++ float overload */
    q2 = cosf(lati - latj);
    q3 = cosf(lati + latj);
    return (int)(6378.388 * acos(0.5 * ((1.0 + q1) * q2 - (1.0 - q1) * q3)) + 1.0);
}

static int dist_att(const float *x, const float *y, int i, int j)
{ /* vrpHelper.cpp:138-158 */
    float xd = x[i] - x[j];
    float yd = y[i] - y[j];
    float rij = sqrt((xd * xd + yd * yd) / 10.0);
    float tij = dtrunc_(rij);
    return tij < rij ? (int)tij + 1 : (int)tij;
}

/* compute_distances, vrpHelper.cpp:160-184; dist_type 0=EUC_2D 1=CEIL_2D 2=GEO 3=ATT
 * (DistanceTypeEnum, problem.h:36-38; unknown types fall back to EUC_2D, :56). */
void orc_compute_distances(int n, const float *x, const float *y, int dist_type, float *dist)
{
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) {
            float d;
            switch (dist_type) {
            case 1: d = (float)dist_ceil(x, y, i, j); break;
            case 2: d = (float)dist_geo(x, y, i, j); break;
            case 3: d = (float)dist_att(x, y, i, j); break;
            default: d = dist_euc(x, y, i, j); break;
            }
            dist[(size_t)i * n + j] = d;
        }
}

/* sort2 / swap2: unstable quicksort with a middle pivot, utilities.cpp:230-266.
 * Its tie order decides the NN-list order, so it is restated step for step. */
static void swap2_(float v[], int v2[], int i, int j)
{
    float t1 = v[i]; v[i] = v[j]; v[j] = t1;
    int t2 = v2[i]; v2[i] = v2[j]; v2[j] = t2;
}

static void sort2_(float v[], int v2[], int left, int right)
{
    int k, last;
    if (left >= right) return;
    swap2_(v, v2, left, (left + right) / 2);
    last = left;
    for (k = left + 1; k <= right; k++)
        if (v[k] < v[left]) swap2_(v, v2, ++last, k);
    swap2_(v, v2, left, last);
    sort2_(v, v2, left, last);
    sort2_(v, v2, last + 1, right);
}

/* compute_nn_lists, vrpHelper.cpp:188-236: depth nn = max(nn_ls, nn_ants) clamped
 * to n-1; self and the depot get INFINITY so they sort last.  Returns nn. */
int orc_compute_nn_lists(int n, const float *dist, int nn_ls, int nn_ants, int *nn_out)
{
    int nn = nn_ls >= nn_ants ? nn_ls : nn_ants;
    if (nn >= n) nn = n - 1;
    float *dv = (float *)malloc(sizeof(float) * n);
    int *hv = (int *)malloc(sizeof(int) * n);
    for (int node = 0; node < n; node++) {
        for (int i = 0; i < n; i++) {
            dv[i] = dist[(size_t)node * n + i];
            hv[i] = i;
        }
        dv[node] = INFINITY;
        dv[0] = INFINITY;
        sort2_(dv, hv, 0, n - 1);
        for (int i = 0; i < nn; i++) nn_out[(size_t)node * nn + i] = hv[i];
    }
    free(dv);
    free(hv);
    return nn;
}

/* compute_tour_length, vrpHelper.cpp:244-253 (fp32 sum in tour order). */
float orc_tour_length(int n, const float *dist, const int *tour, int tour_size)
{
    float len = 0;
    for (int i = 0; i < tour_size - 1; i++) len += dist[(size_t)tour[i] * n + tour[i + 1]];
    return len;
}

/* Same sum in double: the FP64 recheck of every reported cost. */
double orc_tour_length_f64(int n, const float *dist, const int *tour, int tour_size)
{
    double len = 0;
    for (int i = 0; i < tour_size - 1; i++) len += (double)dist[(size_t)tour[i] * n + tour[i + 1]];
    return len;
}

/* check_solution + check_route, problem.cpp:226-319.  Returns 1 if valid. */
int orc_check_solution(int n, const float *dist, const int *demand, int capacity,
                       float max_dist, float serv_time, const int *tour, int tour_size)
{
    if (tour_size < 2 || tour[0] != 0) return 0;
    int *used = (int *)calloc(n, sizeof(int));
    int ok = 1, route_beg = 0;
    used[0] = 1;
    for (int i = 1; i < tour_size && ok; i++) {
        int c = tour[i];
        if (c < 0 || c >= n) { ok = 0; break; }
        if (c != 0) {
            if (used[c]) ok = 0; else used[c] = 1;
        } else {
            /* check_route(rbeg = route_beg, rend = i), problem.cpp:287-319 */
            if (i - route_beg < 2) { ok = 0; break; }
            int load = 0;
            for (int k = route_beg + 1; k < i; k++) load += demand[tour[k]];
            if (load > capacity) { ok = 0; break; }
            float d = orc_tour_length(n, dist, tour + route_beg, i - route_beg + 1);
            d += serv_time * (i - route_beg - 1);
            if (d > max_dist) { ok = 0; break; }
            route_beg = i;
        }
    }
    for (int i = 0; i < n && ok; i++) if (!used[i]) ok = 0;
    free(used);
    return ok;
}

/* Leaf order of the I-Roulette tournament (kernel.cl:340-366): simulating the
 * rounds with list concatenation gives, for every node, the rank at which it
 * wins ties (smaller = preferred).  prio[node] = rank. */
void orc_tournament_priority(int n, int *prio)
{
    /* lists stored as linked chains: head[i], tail[i], next[node] */
    int *head = (int *)malloc(sizeof(int) * n), *tail = (int *)malloc(sizeof(int) * n);
    int *next = (int *)malloc(sizeof(int) * n);
    for (int i = 0; i < n; i++) { head[i] = tail[i] = i; next[i] = -1; }
    int offset = n;
    while (offset > 0) {
        if (offset % 2 != 0 && offset - 1 != 0) {
            int o = offset - 1;
            next[tail[0]] = head[o]; tail[0] = tail[o];
        }
        offset /= 2;
        for (int i = 0; i < offset; i++) {
            next[tail[i]] = head[i + offset]; tail[i] = tail[i + offset];
        }
    }
    int rank = 0;
    for (int v = (n > 0 ? head[0] : -1); v >= 0; v = next[v]) prio[v] = rank++;
    free(head); free(tail); free(next);
}

/* pow(x, e) rule for total_info (kernel.cl:678,788): exact left-to-right
 * products for small non-negative integer exponents, powf otherwise. */
float orc_pow_rule(float x, float e)
{
    if (e == 1.0f) return x;
    if (e >= 0.0f && e <= 8.0f && e == (float)(int)e) {
        int k = (int)e;
        if (k == 0) return 1.0f;
        float r = x;
        for (int i = 1; i < k; i++) r = r * x;
        return r;
    }
    return powf(x, e);
}

/* ---------------------------------------------------------------------- */
/* construct_solution + independent_roulette (kernel.cl:325-373, 382-493)  */
/* ---------------------------------------------------------------------- */
typedef struct construct_ws {
    float *dist0, *ti, *dw, *prob;
    int *scratch_idx;
    unsigned char *visited, *cand;
} construct_ws;

static void ws_alloc(construct_ws *w, int n)
{
    w->dist0 = (float *)malloc(sizeof(float) * n);
    w->ti = (float *)malloc(sizeof(float) * n);
    w->dw = (float *)malloc(sizeof(float) * n);
    w->prob = (float *)malloc(sizeof(float) * n);
    w->scratch_idx = (int *)malloc(sizeof(int) * n);
    w->visited = (unsigned char *)malloc(n);
    w->cand = (unsigned char *)malloc(n);
}

static void ws_free(construct_ws *w)
{
    free(w->dist0); free(w->ti); free(w->dw); free(w->prob);
    free(w->scratch_idx); free(w->visited); free(w->cand);
}

/* One ant: one OpenCL work-group of nloc work-items, emulated phase by phase. */
static int construct_one(const orc_state *s, int ant, construct_ws *w)
{
    const int n = s->n, nloc = s->nloc, T = 2 * n;
    int *seeds = s->seeds + (size_t)ant * nloc;
    int *tour = s->solutions + (size_t)ant * T;
    const float *dist = s->dist, *total = s->total;
    int status = ORC_OK;

    for (int i = 0; i < n; i++) { /* kernel.cl:402-407 */
        w->dist0[i] = dist[(size_t)i * n];
        w->visited[i] = 0;
    }
    int route_load = 0, step = 0, visited_cnt = 1, cur = 0;
    float route_dist = 0, tour_dist = 0;
    w->visited[0] = 1; /* kernel.cl:424-435 */
    tour[0] = 0;

    while (visited_cnt < n) { /* kernel.cl:438 */
        if (step >= T - 3) { status = ORC_ERR_STEP_LIMIT; break; }
        for (int i = 0; i < n; i++) { /* kernel.cl:440-452 */
            w->ti[i] = total[(size_t)cur * n + i];
            w->dw[i] = dist[(size_t)cur * n + i];
        }
        for (int i = 0; i < n; i++) {
            w->cand[i] = 0;
            if (w->visited[i] == 0 && route_load + s->demand[i] <= s->capacity &&
                route_dist + (w->dw[i] + s->serv_time) + w->dist0[i] <= s->max_dist)
                w->cand[i] = 1;
        }
        /* independent_roulette, kernel.cl:331-337: lane l draws for i = l, l+nloc, ... */
        for (int l = 0; l < nloc; l++)
            for (int i = l; i < n; i += nloc) {
                float r = orc_ran01(&seeds[l]) + 0.001f;
                float p = w->ti[i] * 100;
                float c = (float)w->cand[i];
                w->prob[i] = r * p * c;
                w->scratch_idx[i] = i;
            }
        /* tournament, kernel.cl:343-366 */
        int offset = n;
        while (offset > 0) {
            if (offset % 2 != 0) {
                float mine = w->prob[0], other = w->prob[offset - 1];
                if (other > mine) { w->prob[0] = other; w->scratch_idx[0] = w->scratch_idx[offset - 1]; }
            }
            offset /= 2;
            for (int i = 0; i < offset; i++) {
                float other = w->prob[i + offset], mine = w->prob[i];
                if (other > mine) { w->prob[i] = other; w->scratch_idx[i] = w->scratch_idx[i + offset]; }
            }
        }
        /* queen ant moves, kernel.cl:458-477 */
        int nxt;
        step++;
        if (w->prob[0] == 0) {
            nxt = 0; route_load = 0; route_dist = 0;
        } else {
            nxt = w->scratch_idx[0];
            route_load += s->demand[nxt];
            route_dist += w->dw[nxt] + s->serv_time;
            visited_cnt++;
        }
        w->visited[nxt] = 1;
        tour[step] = nxt;
        tour_dist += w->dw[nxt];
        cur = nxt;
    }
    if (status != ORC_OK) {
        tour[T - 1] = 0;
        s->lens[ant] = INFINITY;
        return status;
    }
    tour_dist += w->dist0[tour[step]]; /* kernel.cl:482-488 */
    step++;
    tour[step] = 0;
    tour[T - 1] = step + 1;
    s->lens[ant] = tour_dist;
    return ORC_OK;
}

/* Ant-parallel driver: n_threads POSIX threads pull ant indices from a shared
 * counter (each ant is independent: its own lane seeds, tour and length). */
enum { PAR_CONSTRUCT = 0, PAR_LS = 1, PAR_CONSTRUCT_NN = 2 };
typedef struct par_ctx {
    orc_state *s;
    int kind, K, next, status;
    const int *nnl;
    pthread_mutex_t mu;
} par_ctx;

static int construct_one(const orc_state *s, int ant, construct_ws *w);
struct ls_ws;
static int local_search_one(const orc_state *s, int ant, struct ls_ws *w);
static struct ls_ws *ls_ws_alloc(int n);
static void ls_ws_free(struct ls_ws *w);
static int construct_nn_one(const orc_state *s, int ant, const int *nnl, int K,
                            unsigned char *visited, float *dist0);

static void *par_worker(void *arg)
{
    par_ctx *c = (par_ctx *)arg;
    orc_state *s = c->s;
    int n = s->n, status = ORC_OK;
    construct_ws cw;
    memset(&cw, 0, sizeof cw);
    struct ls_ws *lw = NULL;
    unsigned char *visited = NULL;
    float *dist0 = NULL;
    if (c->kind == PAR_CONSTRUCT) ws_alloc(&cw, n);
    if (c->kind == PAR_LS) lw = ls_ws_alloc(n);
    if (c->kind == PAR_CONSTRUCT_NN) {
        visited = (unsigned char *)malloc(n);
        dist0 = (float *)malloc(sizeof(float) * n);
    }
    for (;;) {
        int a = __atomic_fetch_add(&c->next, 1, __ATOMIC_RELAXED);
        if (a >= s->n_ants) break;
        int st;
        if (c->kind == PAR_CONSTRUCT) st = construct_one(s, a, &cw);
        else if (c->kind == PAR_LS) st = local_search_one(s, a, lw);
        else st = construct_nn_one(s, a, c->nnl, c->K, visited, dist0);
        if (st < status) status = st;
    }
    if (c->kind == PAR_CONSTRUCT) ws_free(&cw);
    if (lw) ls_ws_free(lw);
    free(visited);
    free(dist0);
    pthread_mutex_lock(&c->mu);
    if (status < c->status) c->status = status;
    pthread_mutex_unlock(&c->mu);
    return NULL;
}

static int par_run(orc_state *s, int kind, const int *nnl, int K, int n_threads)
{
    par_ctx c;
    c.s = s; c.kind = kind; c.K = K; c.next = 0; c.status = ORC_OK; c.nnl = nnl;
    pthread_mutex_init(&c.mu, NULL);
    if (n_threads < 1) n_threads = 1;
    if (n_threads > 256) n_threads = 256;
    if (n_threads == 1) {
        par_worker(&c);
    } else {
        pthread_t th[256];
        for (int t = 0; t < n_threads; t++) pthread_create(&th[t], NULL, par_worker, &c);
        for (int t = 0; t < n_threads; t++) pthread_join(th[t], NULL);
    }
    pthread_mutex_destroy(&c.mu);
    if (c.status < s->status) s->status = c.status;
    return c.status;
}

int orc_construct(orc_state *s, int n_threads) { return par_run(s, PAR_CONSTRUCT, NULL, 0, n_threads); }

/* ---------------------------------------------------------------------- */
/* local_search: two_opt_single_route / two_opt_solution / local_search    */
/* (kernel.cl:126-319, 500-539)                                            */
/* ---------------------------------------------------------------------- */
typedef struct ls_ws {
    int *tour_wrk, *pos;
    float *dist_tour_wrk;
    unsigned char *dlb, *route_map;
} ls_ws;

static ls_ws *ls_ws_alloc(int n)
{
    ls_ws *w = (ls_ws *)malloc(sizeof(ls_ws));
    w->tour_wrk = (int *)malloc(sizeof(int) * 2 * n);
    w->pos = (int *)malloc(sizeof(int) * n);
    w->dist_tour_wrk = (float *)malloc(sizeof(float) * 2 * n);
    w->dlb = (unsigned char *)malloc(n);
    w->route_map = (unsigned char *)malloc(n);
    return w;
}

static void ls_ws_free(ls_ws *w)
{
    free(w->tour_wrk); free(w->pos); free(w->dist_tour_wrk); free(w->dlb); free(w->route_map);
    free(w);
}

static int two_opt_single_route(const orc_state *s, int *tour, int rbeg, int rend,
                                unsigned char *dlb, const unsigned char *route_node_map,
                                int *tour_node_pos, float *dist_tour_wrk)
{
    const int n = s->n, nn_ls = s->nn_ls;
    const float *D = s->dist;
    const int *nn_list = s->nn_list;
    int num_route_node = rend - rbeg + 1;
    int n1, n2, s_n1, s_n2, p_n1, p_n2, pos_n1, pos_n2, i, j, h, l, help;
    int h1 = 0, h2 = 0, h3 = 0, h4 = 0, imp_flag = 1, passes = 0;
    float radius, gain;

    while (imp_flag) { /* kernel.cl:157 */
        if (s->step_limit_passes > 0 && passes >= s->step_limit_passes) return ORC_ERR_LS_LIMIT;
        passes++;
        imp_flag = 0;
        for (l = 0; l < num_route_node; l++) {
            pos_n1 = rbeg + l; /* sequence order, kernel.cl:164 */
            n1 = tour[pos_n1];
            if (dlb[n1]) continue;
            s_n1 = pos_n1 == rend ? tour[rbeg] : tour[pos_n1 + 1];
            radius = D[(size_t)n1 * n + s_n1];
            /* successor search, kernel.cl:180-198 */
            for (h = 0; h < nn_ls; h++) {
                n2 = nn_list[(size_t)n1 * nn_ls + h];
                if (route_node_map[n2] == 0) continue;
                if (radius - D[(size_t)n1 * n + n2] > EPSILON) {
                    pos_n2 = tour_node_pos[n2];
                    s_n2 = pos_n2 == rend ? tour[rbeg] : tour[pos_n2 + 1];
                    gain = -radius + D[(size_t)n1 * n + n2] + D[(size_t)s_n1 * n + s_n2] - dist_tour_wrk[pos_n2];
                    if (gain < -EPSILON) { h1 = n1; h2 = s_n1; h3 = n2; h4 = s_n2; goto exchange2opt; }
                } else break;
            }
            /* predecessor search, kernel.cl:202-230 */
            p_n1 = pos_n1 == rbeg ? tour[rend] : tour[pos_n1 - 1];
            radius = D[(size_t)p_n1 * n + n1];
            for (h = 0; h < nn_ls; h++) {
                n2 = nn_list[(size_t)n1 * nn_ls + h];
                if (route_node_map[n2] == 0) continue;
                if (radius - D[(size_t)n1 * n + n2] > EPSILON) {
                    pos_n2 = tour_node_pos[n2];
                    p_n2 = pos_n2 == rbeg ? tour[rend] : tour[pos_n2 - 1];
                    if (p_n2 == n1 || p_n1 == n2) continue;
                    gain = -radius + D[(size_t)n1 * n + n2] + D[(size_t)p_n1 * n + p_n2] - dist_tour_wrk[pos_n2 - 1];
                    if (gain < -EPSILON) { h1 = p_n1; h2 = n1; h3 = p_n2; h4 = n2; goto exchange2opt; }
                } else break;
            }
            dlb[n1] = 1; /* kernel.cl:232 */
            continue;
        exchange2opt: /* kernel.cl:235-270 */
            imp_flag = 1;
            dlb[h1] = 0; dlb[h2] = 0; dlb[h3] = 0; dlb[h4] = 0;
            if (tour_node_pos[h3] < tour_node_pos[h1]) {
                help = h1; h1 = h3; h3 = help;
                help = h2; h2 = h4; h4 = help;
            }
            i = tour_node_pos[h1];
            j = tour_node_pos[h3];
            dist_tour_wrk[i] = D[(size_t)h1 * n + h3];
            dist_tour_wrk[j] = D[(size_t)h2 * n + h4];
            i++; j--;
            while (i < j) {
                float tmp = dist_tour_wrk[i]; dist_tour_wrk[i] = dist_tour_wrk[j]; dist_tour_wrk[j] = tmp;
                i++; j--;
            }
            i = tour_node_pos[h2];
            j = tour_node_pos[h3];
            while (i < j) {
                n1 = tour[i]; n2 = tour[j];
                tour[i] = n2; tour[j] = n1;
                tour_node_pos[n1] = j; tour_node_pos[n2] = i;
                i++; j--;
            }
        }
    }
    return ORC_OK;
}

/* LocalSearch::swap (localSearch.cpp:301-410): first-improvement exchange of
 * two customers, scanned i < j over tour positions; after an accepted swap the
 * scan resumes at the same i (the reference's `i--`).  Float expressions keep
 * the reference's evaluation order.  Returns the number of swaps applied, or
 * -1 once more than max_swaps (> 0) were applied. */
int orc_swap(int n, const float *dist, const int *demand, int capacity, float max_dist, float serv_time,
             int *tour, int tour_size, int max_swaps)
{
    int *route_load = (int *)malloc(sizeof(int) * (size_t)(n > 1 ? n - 1 : 1));
    float *route_dist = (float *)malloc(sizeof(float) * (size_t)(n > 1 ? n - 1 : 1));
#define D(a, b) dist[(size_t)(a) * n + (b)]
    int load = 0, k = 0, beg = 0, swaps = 0;
    float dd = 0;
    for (int i = 1; i < tour_size; i++) { /* step 1: route loads and lengths */
        load += demand[tour[i]];
        dd += D(tour[i - 1], tour[i]);
        if (tour[i] == 0) {
            route_load[k] = load;
            route_dist[k] = dd + serv_time * (float)(i - beg - 1);
            k++;
            load = 0;
            dd = 0;
            beg = i;
        }
    }
    int p1 = 0;
    for (int i = 1; i < tour_size; i++) { /* step 2 */
        const int n1 = tour[i];
        if (n1 == 0) {
            p1++;
            continue;
        }
        const int p_n1 = tour[i - 1], s_n1 = tour[i + 1];
        int p2 = p1;
        for (int j = i + 1; j < tour_size; j++) {
            const int n2 = tour[j];
            if (n2 == 0) {
                p2++;
                continue;
            }
            const int p_n2 = tour[j - 1], s_n2 = tour[j + 1];
            float gain;
            if (j == i + 1)
                gain = -(D(p_n1, n1) + D(n2, s_n2)) + (D(p_n1, n2) + D(n1, s_n2));
            else
                gain = -(D(p_n1, n1) + D(n1, s_n1) + D(p_n2, n2) + D(n2, s_n2)) +
                       (D(p_n1, n2) + D(n2, s_n1) + D(p_n2, n1) + D(n1, s_n2));
            if (!(gain < -EPSILON)) continue;
            int load1, load2;
            float dist1, dist2;
            if (p1 != p2) {
                load1 = route_load[p1] - demand[n1] + demand[n2];
                load2 = route_load[p2] - demand[n2] + demand[n1];
                dist1 = route_dist[p1] - (D(p_n1, n1) + D(n1, s_n1)) + (D(p_n1, n2) + D(n2, s_n1));
                dist2 = route_dist[p2] - (D(p_n2, n2) + D(n2, s_n2)) + (D(p_n2, n1) + D(n1, s_n2));
                if ((load1 > capacity || load2 > capacity) || (dist1 > max_dist || dist2 > max_dist)) continue;
            } else {
                load1 = route_load[p1];
                load2 = load1;
                dist1 = route_dist[p1] + gain;
                dist2 = dist1;
            }
            tour[i] = n2;
            tour[j] = n1;
            route_load[p1] = load1;
            route_load[p2] = load2;
            route_dist[p1] = dist1;
            route_dist[p2] = dist2;
            if (++swaps > max_swaps && max_swaps > 0) {
                free(route_load);
                free(route_dist);
                return -1;
            }
            i--;
            break;
        }
    }
#undef D
    free(route_load);
    free(route_dist);
    return swaps;
}

static int local_search_one(const orc_state *s, int ant, ls_ws *w)
{
    const int n = s->n, T = 2 * n;
    int *tour = s->solutions + (size_t)ant * T;
    int tour_size = tour[T - 1];
    int status = ORC_OK;
    if (tour_size < 2) return ORC_OK; /* failed construct: nothing to improve */
    for (int i = 0; i < tour_size; i++) w->tour_wrk[i] = tour[i]; /* kernel.cl:517-523 */
    for (int i = 0; i < tour_size - 1; i++)
        w->dist_tour_wrk[i] = s->dist[(size_t)w->tour_wrk[i] * n + w->tour_wrk[i + 1]];
    /* two_opt_solution, kernel.cl:279-319 */
    for (int i = 0; i < n; i++) { w->dlb[i] = 0; w->route_map[i] = 0; }
    for (int j = 0; j < tour_size; j++) w->pos[w->tour_wrk[j]] = j;
    int route_beg = 0;
    for (int i = 1; i < tour_size; i++) {
        if (w->tour_wrk[i] == 0) {
            w->pos[0] = route_beg;
            int st = two_opt_single_route(s, w->tour_wrk, route_beg, i - 1, w->dlb, w->route_map,
                                          w->pos, w->dist_tour_wrk);
            if (st < status) status = st;
            for (int j = 0; j < n; j++) w->route_map[j] = 0;
            route_beg = i;
        } else {
            w->route_map[w->tour_wrk[i]] = 1;
        }
    }
    for (int i = 0; i < tour_size; i++) tour[i] = w->tour_wrk[i]; /* kernel.cl:530-538 */
    float len = 0;
    if (s->ls_flag & 2) { /* second stage: swap, then compute_tour_length (localSearch.cpp:63-70) */
        const int sw = orc_swap(n, s->dist, s->demand, s->capacity, s->max_dist, s->serv_time, tour, tour_size,
                                ORC_SWAP_LIMIT_PER_NODE * n);
        if (sw < 0 && ORC_ERR_LS_LIMIT < status) status = ORC_ERR_LS_LIMIT;
        for (int i = 0; i < tour_size - 1; i++) len += s->dist[(size_t)tour[i] * n + tour[i + 1]];
    } else {
        for (int i = 0; i < tour_size - 1; i++) len += w->dist_tour_wrk[i];
    }
    s->lens[ant] = len;
    return status;
}

int orc_local_search(orc_state *s, int n_threads) { return par_run(s, PAR_LS, NULL, 0, n_threads); }

/* ---------------------------------------------------------------------- */
/* Statistics: best_solution_phase_0/1 (kernel.cl:594-665),               */
/* find_best_solution (g_aco.cpp:419-490), update_best_so_far (kernel.cl:546-586) */
/* ---------------------------------------------------------------------- */
void orc_find_best(orc_state *s)
{
    const int A = s->n_ants, T = 2 * s->n, grp = s->nloc; /* grp_size = mwg/4 = nloc */
    const int num_grps = (A + grp - 1) / grp;
    float *sv = (float *)calloc(grp, sizeof(float));
    int *si = (int *)malloc(sizeof(int) * grp);
    float minval = INFINITY;
    int minidx = 0;
    for (int g = 0; g < num_grps; g++) {
        for (int lid = 0; lid < grp; lid++) {
            int gid = g * grp + lid;
            sv[lid] = gid < A ? s->lens[gid] : INFINITY;
            si[lid] = gid;
        }
        for (int offset = grp / 2; offset > 0; offset /= 2)
            for (int lid = 0; lid < offset; lid++) {
                float other = sv[lid + offset], mine = sv[lid];
                if (other < mine) { sv[lid] = other; si[lid] = si[lid + offset]; }
            }
        /* phase 1: serial scan over groups with strict < (kernel.cl:645-654) */
        if (g == 0) { minval = sv[0]; minidx = si[0]; }
        else if (sv[0] < minval) { minval = sv[0]; minidx = si[0]; }
    }
    free(sv); free(si);
    s->solutions[(size_t)T * (A + 1)] = minidx;
    s->update_flag = (minval - s->lens[A] < -EPSILON) ? 1 : 0;
}

void orc_update_best_so_far(orc_state *s, float time)
{
    if (!s->update_flag) return;
    const int A = s->n_ants, T = 2 * s->n;
    int idx = s->solutions[(size_t)T * (A + 1)];
    const int *it = s->solutions + (size_t)T * idx;
    int *best = s->solutions + (size_t)T * A;
    int size = it[T - 1];
    float len = s->lens[idx];
    for (int g = 0; g < size; g++) best[g] = it[g];
    best[T - 1] = size;
    s->lens[A] = len;
    if (s->num_bsf < s->record_cap) {
        s->records[s->num_bsf].iter = s->iteration;
        s->records[s->num_bsf].length = len;
        s->records[s->num_bsf].time = time;
    }
    s->num_bsf++;
}

/* get_elites, kernel.cl:717-741 */
void orc_get_elites(orc_state *s)
{
    const int A = s->n_ants;
    float *help_b = (float *)malloc(sizeof(float) * (A > 0 ? A : 1));
    s->elites[0] = A;
    for (int k = 0; k < A; k++) help_b[k] = s->lens[k];
    for (int i = 0; i < s->ras_ranks - 1; i++) {
        float b = help_b[0];
        int target = 0;
        for (int k = 0; k < A; k++)
            if (help_b[k] < b) { b = help_b[k]; target = k; }
        help_b[target] = INFINITY;
        s->elites[i + 1] = target;
    }
    free(help_b);
}

/* pheromone_init, kernel.cl:672-679 */
void orc_pheromone_init(orc_state *s, float trail)
{
    size_t nn = (size_t)s->n * s->n;
    for (size_t g = 0; g < nn; g++) {
        s->tau[g] = trail;
        s->total[g] = orc_pow_rule(s->tau[g], s->alpha) * orc_pow_rule(1.0f / (s->dist[g] + 0.1f), s->beta);
    }
}

/* pheromone_evaporation, kernel.cl:685-692 */
void orc_pheromone_evaporation(orc_state *s)
{
    size_t nn = (size_t)s->n * s->n;
    float f = 1.0f - s->rho;
    for (size_t g = 0; g < nn; g++) s->tau[g] = f * s->tau[g];
}

/* pheromone_deposit, kernel.cl:747-776, applied in the canonical order:
 * elite 0..ras_ranks-1, tour positions ascending (the reference's CAS atomics
 * leave the order unspecified). */
void orc_pheromone_deposit(orc_state *s)
{
    const int n = s->n, T = 2 * n;
    for (int grp = 0; grp < s->ras_ranks; grp++) {
        int tid = s->elites[grp];
        const int *tour = s->solutions + (size_t)tid * T;
        int tour_size = tour[T - 1];
        float tour_length = s->lens[tid];
        int weight = s->ras_ranks - grp;
        float d_tau = 1.0f * weight / tour_length;
        for (int i = 0; i < tour_size - 1; i++)
            s->tau[(size_t)tour[i] * n + tour[i + 1]] += d_tau;
    }
}

/* compute_total_info, kernel.cl:782-789 */
void orc_compute_total_info(orc_state *s)
{
    size_t nn = (size_t)s->n * s->n;
    for (size_t g = 0; g < nn; g++)
        s->total[g] = orc_pow_rule(s->tau[g], s->alpha) * orc_pow_rule(1.0f / (s->dist[g] + 0.1f), s->beta);
}

/* g_ACO::init_aco, g_aco.cpp:63-93 (local search after the bootstrap construct
 * when ls_flag is set: the call commented out at :84-86). */
int orc_init_aco(orc_state *s, int n_threads)
{
    const int A = s->n_ants;
    s->iteration = 0;
    s->num_bsf = 0;
    s->status = ORC_OK;
    s->lens[A] = INFINITY; /* g_aco.cpp:660-665 */
    orc_pheromone_init(s, 0.5f);
    int st = orc_construct(s, n_threads);
    if (st == ORC_OK && s->ls_flag) st = orc_local_search(s, n_threads);
    orc_find_best(s);
    orc_update_best_so_far(s, 0.0f);
    float trail_0 = 1.0f / ((s->rho) * s->lens[A]);
    orc_pheromone_init(s, trail_0);
    s->iteration++;
    return st;
}

/* g_ACO::run_aco_iteration + pheromone_update (g_aco.cpp:122-134, 233-243) and
 * the iteration++ of main.cpp:86. */
/* The random-descent stage: every ant's tour takes ns_rounds NeighbourSearch
 * proposals (ns_oracle.c), the valid improving ones applied, then its length is
 * recomputed as compute_tour_length sums it (vrpHelper.cpp:244-253). */
static void ns_stage(orc_state *s)
{
    const int n = s->n, T = 2 * n;
    for (int a = 0; a < s->n_ants; a++) {
        int *tour = s->solutions + (size_t)a * T;
        const int size = tour[T - 1];
        if (size < 2) continue;
        orc_ns_descent(n, s->dist, s->demand, s->capacity, s->max_dist, s->serv_time, tour, size,
                       orc_ns_seed(s->ns_seed, s->iteration, a), s->ns_rounds);
        float len = 0;
        for (int i = 0; i < size - 1; i++) len += s->dist[(size_t)tour[i] * n + tour[i + 1]];
        s->lens[a] = len;
    }
}

int orc_run_aco_iteration(orc_state *s, int n_threads)
{
    int st = orc_construct(s, n_threads);
    if (st == ORC_OK && s->ls_flag) st = orc_local_search(s, n_threads);
    if (st == ORC_OK && s->ns_rounds > 0) ns_stage(s);
    orc_find_best(s);
    orc_update_best_so_far(s, 0.0f);
    orc_pheromone_evaporation(s);
    orc_get_elites(s);
    orc_pheromone_deposit(s);
    orc_compute_total_info(s);
    s->iteration++;
    return st;
}

/* ---------------------------------------------------------------------- */
/* Throughput mode: this project's candidate-list sampler (no reference    */
/* counterpart).  Lane j (0..31) of an ant owns its Park-Miller state j and */
/* draws u_j every step; the first nn_ants entries of the NN list are the  */
/* candidates, and the feasible one with the smallest -ln(u_j) /          */
/* choice_info wins (exponential race: the roulette's probabilities),      */
/* keyed as the device does it; full-row argmax fallback over all feasible */
/* customers when no candidate has weight; depot return otherwise.         */
/* ---------------------------------------------------------------------- */
static float f_of_bits(uint32_t b) { float f; memcpy(&f, &b, 4); return f; }
static uint32_t bits_of_f(float f) { uint32_t b; memcpy(&b, &f, 4); return b; }

/* E = -ln(u): u = m*2^e, m in [sqrt(1/2), sqrt(2)), t = m - 1,
 * ln(m) = t + t^2*Q(t), Q the degree-6 least-squares fit on Chebyshev nodes --
 * the device's race_exp1 operation for operation (Horner with fmaf). */
float orc_race_exp1(float u)
{
    const uint32_t b = bits_of_f(u);
    int e = (int)(b >> 23) - 127;
    float m = f_of_bits((b & 0x007fffffu) | 0x3f800000u);
    if (m > 1.41421354f) { m = m * 0.5f; e += 1; }
    const float t = m - 1.0f;
    float q = fmaf(-0.098038554f, t, 0.16080461f);
    q = fmaf(q, t, -0.172902f);
    q = fmaf(q, t, 0.19920385f);
    q = fmaf(q, t, -0.24968483f);
    q = fmaf(q, t, 0.333343f);
    q = fmaf(q, t, -0.5000038f);
    const float tq = t * q;
    const float lm = fmaf(t, tq, t);
    return 0.0f - fmaf((float)e, 0.693147182f, lm);
}

/* The device's race_key: bits of E * (1/w), low 5 bits = lane; the smallest wins. */
#define RACE_NO_KEY 0xffffffffu
static uint32_t race_key(float e, float winv, int lane)
{
    return (bits_of_f(e * winv) & ~31u) | (uint32_t)lane;
}

static int construct_nn_one(const orc_state *s, int ant, const int *nnl, int K,
                            unsigned char *visited, float *dist0)
{
    const int n = s->n, T = 2 * n;
    int *seed = s->seeds + (size_t)ant * s->nloc;
    int *tour = s->solutions + (size_t)ant * T;
    const float *dist = s->dist, *total = s->total;
    for (int i = 0; i < n; i++) { dist0[i] = dist[(size_t)i * n]; visited[i] = 0; }
    int route_load = 0, step = 0, visited_cnt = 1, cur = 0;
    float route_dist = 0, tour_dist = 0;
    visited[0] = 1;
    tour[0] = 0;
    while (visited_cnt < n) {
        if (step >= T - 3) { tour[T - 1] = 0; s->lens[ant] = INFINITY; return ORC_ERR_STEP_LIMIT; }
        float u[32];
        for (int j = 0; j < 32; j++) u[j] = orc_ran01(&seed[j]);
        uint32_t hk = RACE_NO_KEY;
        int nxt = -1;
        for (int j = 0; j < K; j++) {
            const int c = nnl[(size_t)cur * K + j];
            const float dc = dist[(size_t)cur * n + c];
            const float winv = 1.0f / total[(size_t)cur * n + c]; /* the candidate table's reciprocal weight */
            if (!visited[c] && route_load + s->demand[c] <= s->capacity &&
                route_dist + (dc + s->serv_time) + dist0[c] <= s->max_dist && winv < INFINITY) {
                const uint32_t key = race_key(orc_race_exp1(u[j]), winv, j);
                if (key < hk) { hk = key; nxt = c; }
            }
        }
        if (hk == RACE_NO_KEY) {
            float bv = -1.0f;
            for (int i = 1; i < n; i++) {
                const float di = dist[(size_t)cur * n + i];
                if (!visited[i] && route_load + s->demand[i] <= s->capacity &&
                    route_dist + (di + s->serv_time) + dist0[i] <= s->max_dist) {
                    float v = total[(size_t)cur * n + i];
                    if (v > bv) { bv = v; nxt = i; }
                }
            }
        }
        step++;
        if (nxt < 0) {
            nxt = 0; route_load = 0; route_dist = 0;
        } else {
            route_load += s->demand[nxt];
            route_dist += dist[(size_t)cur * n + nxt] + s->serv_time;
            visited_cnt++;
        }
        visited[nxt] = 1;
        tour[step] = nxt;
        tour_dist += dist[(size_t)cur * n + nxt];
        cur = nxt;
    }
    tour_dist += dist0[tour[step]];
    step++;
    tour[step] = 0;
    tour[T - 1] = step + 1;
    s->lens[ant] = tour_dist;
    return ORC_OK;
}

int orc_construct_nn(orc_state *s, const int *nn_ants_list, int nn_ants, int n_threads)
{
    return par_run(s, PAR_CONSTRUCT_NN, nn_ants_list, nn_ants, n_threads);
}

int orc_init_aco_nn(orc_state *s, const int *nn_ants_list, int nn_ants, int n_threads)
{
    const int A = s->n_ants;
    s->iteration = 0;
    s->num_bsf = 0;
    s->status = ORC_OK;
    s->lens[A] = INFINITY;
    orc_pheromone_init(s, 0.5f);
    int st = orc_construct_nn(s, nn_ants_list, nn_ants, n_threads);
    if (st == ORC_OK && s->ls_flag) st = orc_local_search(s, n_threads);
    orc_find_best(s);
    orc_update_best_so_far(s, 0.0f);
    float trail_0 = 1.0f / ((s->rho) * s->lens[A]);
    orc_pheromone_init(s, trail_0);
    s->iteration++;
    return st;
}

int orc_run_aco_iteration_nn(orc_state *s, const int *nn_ants_list, int nn_ants, int n_threads)
{
    int st = orc_construct_nn(s, nn_ants_list, nn_ants, n_threads);
    if (st == ORC_OK && s->ls_flag) st = orc_local_search(s, n_threads);
    if (st == ORC_OK && s->ns_rounds > 0) ns_stage(s);
    orc_find_best(s);
    orc_update_best_so_far(s, 0.0f);
    orc_pheromone_evaporation(s);
    orc_get_elites(s);
    orc_pheromone_deposit(s);
    orc_compute_total_info(s);
    s->iteration++;
    return st;
}
