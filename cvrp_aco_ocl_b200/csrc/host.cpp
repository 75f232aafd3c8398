// host.cpp -- the host side of the path: instance reader, distances, NN lists,
// seeds, validation and kernel lookup tables.  Built with -ffp-contract=off so
// every float expression rounds the way the reference's host code does.
#include "host.h"

#include <cctype>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>

#include "../../include/cvrp_aco.h"

namespace aco {

// ---------------------------------------------------------------------------
// VRPLIB reader.  Token-driven like io.cpp:353-483: a header key is a
// whitespace-separated token; "KEY" is followed by a ':' token, "KEY:" is not.
// COMMENT carries the optimum as a float when it parses as one (io.cpp:365-372).
// ---------------------------------------------------------------------------
namespace {
struct Tok {
    const std::string &s;
    size_t p = 0;
    explicit Tok(const std::string &src) : s(src) {}
    void skip_ws() { while (p < s.size() && std::isspace((unsigned char)s[p])) p++; }
    bool word(std::string &out) {
        skip_ws();
        if (p >= s.size()) return false;
        size_t b = p;
        while (p < s.size() && !std::isspace((unsigned char)s[p])) p++;
        out.assign(s, b, p - b);
        return true;
    }
    // fscanf("%f"/"%d") semantics: parse a number at the cursor if there is one;
    // on a matching failure nothing is consumed (besides whitespace).
    bool number(float &v) {
        skip_ws();
        if (p >= s.size()) return false;
        const char *b = s.c_str() + p;
        char *e = nullptr;
        v = std::strtof(b, &e);
        if (e == b) return false;
        p += (size_t)(e - b);
        return true;
    }
    bool integer(long &v) {
        skip_ws();
        if (p >= s.size()) return false;
        const char *b = s.c_str() + p;
        char *e = nullptr;
        v = std::strtol(b, &e, 10);
        if (e == b) return false;
        p += (size_t)(e - b);
        return true;
    }
    void rest_of_line() { while (p < s.size() && s[p] != '\n') p++; }
};

bool parse_dist_type(const std::string &w, int &t)
{
    if (w == "EUC_2D") { t = ACO_DIST_EUC_2D; return true; }
    if (w == "CEIL_2D") { t = ACO_DIST_CEIL_2D; return true; }
    if (w == "GEO") { t = ACO_DIST_GEO; return true; }
    if (w == "ATT") { t = ACO_DIST_ATT; return true; }
    return false;
}
} // namespace

int read_vrplib(const char *path, VrpFile &out, std::string &err)
{
    std::ifstream f(path);
    if (!f.is_open()) { err = "cannot open instance file"; return ACO_ERR_IO; }
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string src = ss.str();
    Tok t(src);
    out = VrpFile();
    out.max_distance = INFINITY; // io.cpp:348-350
    out.service_time = 0;
    out.optimum = 0;
    std::string w;
    float dv;
    long lv;
    for (;;) {
        if (!t.word(w)) { err = "NODE_COORD_SECTION not found"; return ACO_ERR_IO; }
        if (w == "NODE_COORD_SECTION") break;
        if (w == "NAME") { t.word(w); t.word(out.name); }
        else if (w == "NAME:") { t.word(out.name); }
        else if (w == "COMMENT" || w == "COMMENT:") { if (t.number(dv)) out.optimum = dv; }
        else if (w == "TYPE" || w == "TYPE:") {
            if (w == "TYPE") t.word(w);
            t.word(w);
            if (w != "CVRP") { err = "not a CVRP instance"; return ACO_ERR_IO; }
        } else if (w == "DIMENSION" || w == "DIMENSION:") {
            if (w == "DIMENSION") t.word(w);
            if (!t.integer(lv)) { err = "bad DIMENSION"; return ACO_ERR_IO; }
            out.n = (int)lv;
        } else if (w == "DISPLAY_DATA_TYPE" || w == "DISPLAY_DATA_TYPE:") {
            t.rest_of_line();
        } else if (w == "EDGE_WEIGHT_TYPE" || w == "EDGE_WEIGHT_TYPE:") {
            if (w == "EDGE_WEIGHT_TYPE") t.word(w);
            t.word(w);
            int dt;
            if (parse_dist_type(w, dt)) out.dist_type = dt;
            else { err = "EDGE_WEIGHT_TYPE " + w + " not implemented"; return ACO_ERR_IO; }
        } else if (w == "CAPACITY" || w == "CAPACITY:") {
            if (w == "CAPACITY") t.word(w);
            if (!t.integer(lv)) { err = "bad CAPACITY"; return ACO_ERR_IO; }
            out.capacity = (int)lv;
        } else if (w == "DISTANCE" || w == "DISTANCE:") {
            if (t.number(dv)) out.max_distance = dv;
        } else if (w == "SERVICE_TIME" || w == "SERVICE_TIME:") {
            if (t.number(dv)) out.service_time = dv;
        }
    }
    if (out.n <= 0 || out.n > (1 << 20)) { err = "bad DIMENSION"; return ACO_ERR_IO; }
    out.x.resize(out.n);
    out.y.resize(out.n);
    out.demand.resize(out.n);
    for (int i = 0; i < out.n; i++) { // io.cpp:495-501: node ids are read and ignored
        float a, b; // fscanf("%d %f %f"): strtof rounding
        if (!t.integer(lv) || !t.number(a) || !t.number(b)) { err = "bad NODE_COORD_SECTION"; return ACO_ERR_IO; }
        out.x[i] = a;
        out.y[i] = b;
    }
    for (;;) { // io.cpp:504-507 (the reference loops forever at EOF)
        if (!t.word(w)) { err = "DEMAND_SECTION not found"; return ACO_ERR_IO; }
        if (w == "DEMAND_SECTION") break;
    }
    for (int i = 0; i < out.n; i++) {
        long id, d;
        if (!t.integer(id) || !t.integer(d)) { err = "bad DEMAND_SECTION"; return ACO_ERR_IO; }
        out.demand[i] = (int)d;
    }
    return ACO_OK;
}

// ---------------------------------------------------------------------------
// Distances (vrpHelper.cpp:35-158): float variables, the reference's mix of
// float and double operations.
// ---------------------------------------------------------------------------
namespace {
inline float trunc_to_float(float v) { return (float)(int)v; }

float d_euc(const float *x, const float *y, int i, int j)
{
    float dx = x[i] - x[j], dy = y[i] - y[j];
    return sqrtf(dx * dx + dy * dy);
}
int d_ceil(const float *x, const float *y, int i, int j)
{
    float dx = x[i] - x[j], dy = y[i] - y[j];
    return (int)std::ceil(sqrtf(dx * dx + dy * dy));
}
float to_rad(float v)
{
    const double pi = 3.14159265358979323846;
    float deg = trunc_to_float(v);
    float mn = v - deg;
    return (float)(pi * (deg + 5.0 * mn / 3.0) / 180.0);
}
int d_geo(const float *x, const float *y, int i, int j)
{
    float lati = to_rad(x[i]), latj = to_rad(x[j]), longi = to_rad(y[i]), longj = to_rad(y[j]);
    float q1 = (float)std::cos(longi - longj);
    float q2 = (float)std::cos(lati - latj);
    float q3 = (float)std::cos(lati + latj);
    return (int)(6378.388 * std::acos(0.5 * ((1.0 + q1) * q2 - (1.0 - q1) * q3)) + 1.0);
}
int d_att(const float *x, const float *y, int i, int j)
{
    float dx = x[i] - x[j], dy = y[i] - y[j];
    float r = (float)std::sqrt((dx * dx + dy * dy) / 10.0);
    float t = trunc_to_float(r);
    return t < r ? (int)t + 1 : (int)t;
}
} // namespace

float point_distance(const float *x, const float *y, int dist_type, int i, int j)
{
    switch (dist_type) {
    case ACO_DIST_CEIL_2D: return (float)d_ceil(x, y, i, j);
    case ACO_DIST_GEO: return (float)d_geo(x, y, i, j);
    case ACO_DIST_ATT: return (float)d_att(x, y, i, j);
    default: return d_euc(x, y, i, j);
    }
}

void compute_distances(int n, const float *x, const float *y, int dist_type, float *dist)
{
    for (int i = 0; i < n; i++) {
        float *row = dist + (size_t)i * n;
        for (int j = 0; j < n; j++) {
            switch (dist_type) {
            case ACO_DIST_CEIL_2D: row[j] = (float)d_ceil(x, y, i, j); break;
            case ACO_DIST_GEO: row[j] = (float)d_geo(x, y, i, j); break;
            case ACO_DIST_ATT: row[j] = (float)d_att(x, y, i, j); break;
            default: row[j] = d_euc(x, y, i, j); break;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// NN lists.  The order of equal distances is the one the reference's
// quicksort produces (utilities.cpp:246-266: pivot = middle element swapped to
// the left end, Lomuto partition with strict <, recursion on [left, last] and
// [last+1, right]); an explicit stack keeps deep recursion off the C stack.
// ---------------------------------------------------------------------------
// Only positions below `keep` are needed: a range that starts at or beyond it
// is never sorted, which leaves positions [0, keep) exactly as the full sort
// would (the recursion only permutes elements inside disjoint ranges).
namespace {
void quicksort_pairs(float *v, int *idx, int left, int right, int keep, std::vector<std::pair<int, int>> &stack)
{
    stack.clear();
    stack.emplace_back(left, right);
    while (!stack.empty()) {
        auto [l, r] = stack.back();
        stack.pop_back();
        if (l >= r || l >= keep) continue;
        int m = (l + r) / 2;
        std::swap(v[l], v[m]);
        std::swap(idx[l], idx[m]);
        int last = l;
        for (int k = l + 1; k <= r; k++)
            if (v[k] < v[l]) {
                ++last;
                std::swap(v[last], v[k]);
                std::swap(idx[last], idx[k]);
            }
        std::swap(v[l], v[last]);
        std::swap(idx[l], idx[last]);
        // the reference recurses on the left part first; processing order does
        // not change the result since the two ranges are disjoint
        stack.emplace_back(last + 1, r);
        stack.emplace_back(l, last);
    }
}
} // namespace

int compute_nn_lists(int n, const float *dist, int nn_ls, int nn_ants, std::vector<int> &nn)
{
    int depth = nn_ls >= nn_ants ? nn_ls : nn_ants;
    if (depth >= n) depth = n - 1;
    if (depth < 0) depth = 0;
    nn.assign((size_t)n * depth, 0);
    std::vector<float> v(n);
    std::vector<int> idx(n);
    std::vector<std::pair<int, int>> stack;
    for (int node = 0; node < n; node++) {
        for (int i = 0; i < n; i++) {
            v[i] = dist[(size_t)node * n + i];
            idx[i] = i;
        }
        v[node] = INFINITY;
        v[0] = INFINITY;
        quicksort_pairs(v.data(), idx.data(), 0, n - 1, depth, stack);
        for (int i = 0; i < depth; i++) nn[(size_t)node * depth + i] = idx[i];
    }
    return depth;
}

float tour_length32(int n, const float *dist, const int *tour, int tour_size)
{
    float len = 0;
    for (int i = 0; i + 1 < tour_size; i++) len += dist[(size_t)tour[i] * n + tour[i + 1]];
    return len;
}

double tour_length64(int n, const float *dist, const int *tour, int tour_size)
{
    double len = 0;
    for (int i = 0; i + 1 < tour_size; i++) len += (double)dist[(size_t)tour[i] * n + tour[i + 1]];
    return len;
}

bool check_solution(int n, const float *dist, const int *demand, int capacity, float max_dist,
                    float serv_time, const int *tour, int tour_size)
{
    if (tour == nullptr || tour_size < 2 || tour[0] != 0) return false;
    std::vector<char> used(n, 0);
    used[0] = 1;
    int route_beg = 0;
    for (int i = 1; i < tour_size; i++) {
        int c = tour[i];
        if (c < 0 || c >= n) return false;
        if (c != 0) {
            if (used[c]) return false;
            used[c] = 1;
            continue;
        }
        if (i - route_beg < 2) return false; // check_route: rend - rbeg >= 2
        int load = 0;
        for (int k = route_beg + 1; k < i; k++) load += demand[tour[k]];
        if (load > capacity) return false;
        float d = tour_length32(n, dist, tour + route_beg, i - route_beg + 1);
        d += serv_time * (float)(i - route_beg - 1);
        if (d > max_dist) return false;
        route_beg = i;
    }
    for (int i = 0; i < n; i++)
        if (!used[i]) return false;
    return true;
}

// ---------------------------------------------------------------------------
// RNG and seeds
// ---------------------------------------------------------------------------
float ran01(int *idum)
{
    // Schrage's decomposition of 16807 * x mod (2^31 - 1) (utilities.cpp:271-288)
    int k = (*idum) / 127773;
    *idum = 16807 * (*idum - k * 127773) - 2836 * k;
    if (*idum < 0) *idum += 2147483647;
    return (1.0f / 2147483647) * (float)(*idum);
}

namespace {
// fp32 -> int as x86 cvttss2si: NaN and out-of-range values give INT_MIN
int cvt_f32_i32(float v)
{
    if (v != v || v >= 2147483648.0f || v <= -2147483648.0f) return INT_MIN;
    return (int)v;
}
} // namespace

void make_seeds(int seed_time, int *rnd_seed, int n_ants, int nloc, int *seeds)
{
    const float t0 = (float)seed_time;
    const float a = (float)n_ants;
    for (int i = 0, total = n_ants * nloc; i < total; i++) {
        const float m = (float)(i % n_ants);
        const float r = ran01(rnd_seed);
        seeds[i] = cvt_f32_i32(t0 + (m * (m + r)) * a);
    }
}

uint32_t pm_pow(uint64_t e)
{
    uint64_t base = kIA, result = 1;
    while (e) {
        if (e & 1) result = (result * base) % kIM;
        base = (base * base) % kIM;
        e >>= 1;
    }
    return (uint32_t)result;
}

uint32_t pm_normalize(int x)
{
    int64_t r = (int64_t)x % (int64_t)kIM;
    if (r < 0) r += kIM;
    return (uint32_t)r;
}

// ---------------------------------------------------------------------------
// Tournament tie order (kernel.cl:343-366).  The reduction keeps the left
// operand on ties, so the surviving element among equal maxima is the first of
// them in the order obtained by concatenating the merged ranges:
// [0] ++ [offset-1] on odd rounds, then [i] ++ [i + offset/2].
// ---------------------------------------------------------------------------
std::vector<int> tournament_priority(int n)
{
    std::vector<int> head(n), tail(n), next(n, -1), prio(n, 0);
    for (int i = 0; i < n; i++) head[i] = tail[i] = i;
    for (int offset = n; offset > 0;) {
        if ((offset & 1) && offset > 1) {
            next[tail[0]] = head[offset - 1];
            tail[0] = tail[offset - 1];
        }
        offset /= 2;
        for (int i = 0; i < offset; i++) {
            next[tail[i]] = head[i + offset];
            tail[i] = tail[i + offset];
        }
    }
    int rank = 0;
    for (int v = n > 0 ? head[0] : -1; v >= 0; v = next[v]) prio[v] = rank++;
    return prio;
}

} // namespace aco
