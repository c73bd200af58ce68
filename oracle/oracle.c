/*
 * oracle.c — CPU restatement of metalroute's canonical shortest-path semantics.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h).  The product never links this file.
 * Each routine names the reference function it restates (paths relative to the
 * metal-route project root).
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>
#include <unistd.h>

#define NO_PRED 0xFFFFFFFFu
#define CAP 0xFFFFFFFEu

static inline uint32_t sat_add(uint32_t a, uint32_t b) {
    uint32_t s = a + b;
    return s < a ? ORC_MAX : s;
}
static inline uint32_t sat_sub(uint32_t a, uint32_t b) { return a > b ? a - b : 0; }

/* passable_search_cost(edge * enter), negotiated.rs:1171-1173 and
 * isolated_step_cost, crates/mr-metal/src/lib.rs:300-302. */
static inline uint32_t cap_mul(uint32_t e, uint32_t w) {
    uint64_t p = (uint64_t)e * (uint64_t)w;
    return p > (uint64_t)CAP ? CAP : (uint32_t)p;
}

uint32_t orc_edge_cost(double length) {
    double scaled = round(length * 16.0);
    if (!isfinite(scaled) || scaled <= 0.0) return 0;
    if (scaled >= (double)ORC_MAX) return ORC_MAX;
    return (uint32_t)scaled;
}

void orc_axis_edge_costs(const double *lines, uint32_t n_lines, uint32_t count, uint32_t *out) {
    for (uint32_t k = 0; k + 1 < count; ++k) {
        double a = k < n_lines ? lines[k] : (double)k;
        double b = (k + 1) < n_lines ? lines[k + 1] : (double)(k + 1);
        out[k] = orc_edge_cost(fabs(b - a));
    }
}

static uint32_t div_ceil_u32(uint32_t a, uint32_t b) { return a / b + (a % b != 0); }

orc_window orc_net_window(uint32_t w, uint32_t h, uint32_t layers, const orc_net *net) {
    (void)layers;
    uint32_t plane = w * h;
    uint32_t sx = (net->src % plane) % w, sy = (net->src % plane) / w;
    uint32_t dx = (net->dst % plane) % w, dy = (net->dst % plane) / w;
    uint32_t x0 = sx < dx ? sx : dx, y0 = sy < dy ? sy : dy;
    uint32_t x1 = sx > dx ? sx : dx, y1 = sy > dy ? sy : dy;
    for (uint32_t i = 0; i < net->n_pads; ++i) {
        uint32_t p = net->pads[i] % plane;
        uint32_t px = p % w, py = p / w;
        if (px < x0) x0 = px;
        if (py < y0) y0 = py;
        if (px > x1) x1 = px;
        if (py > y1) y1 = py;
    }
    uint32_t span = (x1 - x0) > (y1 - y0) ? (x1 - x0) : (y1 - y0);
    uint32_t m = div_ceil_u32(3 * span, 10);
    uint32_t margin = m > 16 ? m : 16;
    orc_window win;
    win.x0 = x0 > margin ? x0 - margin : 0;
    win.y0 = y0 > margin ? y0 - margin : 0;
    win.x1 = (x1 + margin) < (w ? w - 1 : 0) ? (x1 + margin) : (w ? w - 1 : 0);
    win.y1 = (y1 + margin) < (h ? h - 1 : 0) ? (y1 + margin) : (h ? h - 1 : 0);
    return win;
}

int orc_board_planar_forbidden(const orc_grid *g, uint32_t u, uint32_t v) {
    if (!g->board) return 0;
    uint32_t n = g->w * g->h * g->layers;
    if (u >= n || v >= n) return 1;
    uint32_t plane = g->w * g->h;
    uint32_t ul = u / plane, vl = v / plane;
    uint32_t ur = u % plane, vr = v % plane;
    uint32_t ux = ur % g->w, uy = ur / g->w, vx = vr % g->w, vy = vr / g->w;
    if (ul != vl) return 1;
    uint8_t sb, db;
    if (ux == vx && uy == vy + 1) {
        sb = ORC_BOARD_EDGE_NEG_Y; db = ORC_BOARD_EDGE_POS_Y;
    } else if (uy == vy && ux == vx + 1) {
        sb = ORC_BOARD_EDGE_NEG_X; db = ORC_BOARD_EDGE_POS_X;
    } else if (uy == vy && ux + 1 == vx) {
        sb = ORC_BOARD_EDGE_POS_X; db = ORC_BOARD_EDGE_NEG_X;
    } else if (ux == vx && uy + 1 == vy) {
        sb = ORC_BOARD_EDGE_POS_Y; db = ORC_BOARD_EDGE_NEG_Y;
    } else {
        return 1;
    }
    return (g->board[u] & sb) != 0 || (g->board[v] & db) != 0;
}

/* ------------------------------------------------------------------------ */
/* Sorted cell sets (PadSet / sorted_contains, negotiated.rs:596-640,1379-1381). */

typedef struct {
    uint32_t *v;
    uint32_t n;
} cellset;

static int cmp_u32(const void *a, const void *b) {
    uint32_t x = *(const uint32_t *)a, y = *(const uint32_t *)b;
    return x < y ? -1 : x > y;
}

static cellset cellset_make(const uint32_t *src, uint32_t n) {
    cellset s;
    s.v = (uint32_t *)malloc(sizeof(uint32_t) * (n ? n : 1));
    s.n = 0;
    if (n) {
        memcpy(s.v, src, sizeof(uint32_t) * n);
        qsort(s.v, n, sizeof(uint32_t), cmp_u32);
        uint32_t k = 0;
        for (uint32_t i = 0; i < n; ++i)
            if (k == 0 || s.v[k - 1] != s.v[i]) s.v[k++] = s.v[i];
        s.n = k;
    }
    return s;
}
static void cellset_free(cellset *s) { free(s->v); }
static int cellset_has(const cellset *s, uint32_t c) {
    uint32_t lo = 0, hi = s->n;
    while (lo < hi) {
        uint32_t mid = lo + (hi - lo) / 2;
        if (s->v[mid] < c) lo = mid + 1;
        else hi = mid;
    }
    return lo < s->n && s->v[lo] == c;
}

/* ------------------------------------------------------------------------ */
/* Binary min-heap keyed by (priority, cell): Rust's
 * BinaryHeap<(Reverse<Cost>, Reverse<CellIdx>)> pops the smallest priority and,
 * among ties, the smallest cell (dijkstra.rs:84-87). */

typedef struct {
    uint64_t *a;
    size_t n, cap;
} heap;

static void heap_push(heap *h, uint32_t prio, uint32_t cell) {
    if (h->n == h->cap) {
        h->cap = h->cap ? h->cap * 2 : 1024;
        h->a = (uint64_t *)realloc(h->a, h->cap * sizeof(uint64_t));
    }
    uint64_t key = ((uint64_t)prio << 32) | cell;
    size_t i = h->n++;
    while (i > 0) {
        size_t p = (i - 1) / 2;
        if (h->a[p] <= key) break;
        h->a[i] = h->a[p];
        i = p;
    }
    h->a[i] = key;
}

static int heap_pop(heap *h, uint32_t *prio, uint32_t *cell) {
    if (h->n == 0) return 0;
    uint64_t top = h->a[0];
    uint64_t last = h->a[--h->n];
    size_t i = 0;
    for (;;) {
        size_t l = 2 * i + 1;
        if (l >= h->n) break;
        size_t c = (l + 1 < h->n && h->a[l + 1] < h->a[l]) ? l + 1 : l;
        if (h->a[c] >= last) break;
        h->a[i] = h->a[c];
        i = c;
    }
    if (h->n) h->a[i] = last;
    *prio = (uint32_t)(top >> 32);
    *cell = (uint32_t)top;
    return 1;
}

/* ------------------------------------------------------------------------ */
/* The isolated static cost model of route_legal_once, negotiated.rs:2914-3043,
 * for the alone-path case (no owner, no halo, unoccupied ViaGuard, no locally
 * forbidden via XYs). */

typedef struct {
    const orc_grid *g;
    const orc_edges *e;
    uint32_t src, dst;
    orc_window win;
    cellset pads, via_pads;
    uint32_t plane, n;
    /* heuristic prefix sums (ManhattanCosts, negotiated.rs:1182-1194,1253-1266) */
    uint64_t *xp, *yp;
    int use_h;
    uint32_t via_h_cost;
} iso_ctx;

static int iso_in_window(const iso_ctx *c, uint32_t cell) {
    uint32_t r = cell % c->plane;
    uint32_t x = r % c->g->w, y = r / c->g->w;
    return x >= c->win.x0 && x <= c->win.x1 && y >= c->win.y0 && y <= c->win.y1;
}
static int is_obstacle(const orc_grid *g, uint32_t cell) { return g->cost[cell] == ORC_MAX; }
static int board_trace_forbidden(const orc_grid *g, uint32_t cell) {
    return g->board && (g->board[cell] & ORC_BOARD_TRACE_NODE);
}
static int board_via_forbidden(const orc_grid *g, uint32_t cell) {
    return g->board && (g->board[cell] & ORC_BOARD_VIA_NODE);
}
static int static_via_forbidden(const orc_grid *g, uint32_t cell) {
    return g->via_forbidden && g->via_forbidden[cell];
}

/* blocked_fn, negotiated.rs:2933-2966 */
static int iso_blocked(const iso_ctx *c, uint32_t cell) {
    if (!iso_in_window(c, cell)) return 1;
    if (board_trace_forbidden(c->g, cell)) return 1;
    if (cell == c->src || cell == c->dst) return 0;
    return is_obstacle(c->g, cell) && !cellset_has(&c->pads, cell);
}

/* enter_weight, negotiated.rs:2914-2920 */
static uint32_t iso_enter(const iso_ctx *c, uint32_t cell) {
    if (is_obstacle(c->g, cell) && cellset_has(&c->pads, cell)) return 1;
    return c->g->cost[cell];
}

/* cost_fn, negotiated.rs:2921-2932 (directed superset: a per-edge base price). */
static uint32_t iso_planar_step(const iso_ctx *c, uint32_t u, uint32_t v) {
    if (orc_board_planar_forbidden(c->g, u, v)) return ORC_MAX;
    const orc_grid *g = c->g;
    uint32_t base;
    uint32_t ur = u % c->plane, vr = v % c->plane;
    uint32_t ux = ur % g->w, uy = ur / g->w, vx = vr % g->w, vy = vr / g->w;
    if (c->e->directed) {
        uint32_t dir;
        if (uy + 1 == vy) dir = 0;       /* u is v's -y neighbour */
        else if (ux + 1 == vx) dir = 1;  /* -x */
        else if (ux == vx + 1) dir = 2;  /* +x */
        else dir = 3;                    /* +y */
        base = c->e->directed[(size_t)v * 4 + dir];
        if (base == ORC_MAX) return ORC_MAX;
    } else if (uy == vy) {
        base = c->e->x_edge[ux < vx ? ux : vx];
    } else {
        base = c->e->y_edge[uy < vy ? uy : vy];
    }
    return cap_mul(base, iso_enter(c, v));
}

/* via_step, negotiated.rs:3010-3043 (unoccupied guard: only the static checks). */
static int iso_via_step(const iso_ctx *c, uint32_t u, uint32_t v, uint32_t *step) {
    uint32_t lu = u / c->plane, lv = v / c->plane;
    uint32_t k = lu < lv ? lu : lv;
    if (!c->e->via_allowed || !c->e->via_allowed[k]) return 0;
    if (board_via_forbidden(c->g, u) || board_via_forbidden(c->g, v)) return 0;
    if (static_via_forbidden(c->g, u) && !cellset_has(&c->via_pads, u)) return 0;
    if (static_via_forbidden(c->g, v) && !cellset_has(&c->via_pads, v)) return 0;
    *step = cap_mul(c->e->via_edge[k], iso_enter(c, v));
    return 1;
}

static uint32_t axis_leg(const uint64_t *prefix, uint32_t i, uint32_t j) {
    uint32_t lo = i < j ? i : j, hi = i < j ? j : i;
    uint64_t t = prefix[hi] - prefix[lo];
    return t > ORC_MAX ? ORC_MAX : (uint32_t)t;
}

/* manhattan_scaled, negotiated.rs:1235-1251 */
static uint32_t iso_h(const iso_ctx *c, uint32_t cell) {
    if (!c->use_h) return 0;
    const orc_grid *g = c->g;
    uint32_t ar = cell % c->plane, br = c->dst % c->plane;
    uint32_t planar = sat_add(axis_leg(c->xp, ar % g->w, br % g->w), axis_leg(c->yp, ar / g->w, br / g->w));
    uint32_t la = cell / c->plane, lb = c->dst / c->plane;
    uint32_t dl = la > lb ? la - lb : lb - la;
    uint64_t vm = (uint64_t)dl * c->via_h_cost;
    uint32_t vterm = vm > ORC_MAX ? ORC_MAX : (uint32_t)vm;
    return sat_add(planar, vterm);
}

static void iso_init(iso_ctx *c, const orc_grid *g, const orc_edges *e, const orc_net *net, orc_window win,
                     int use_h, uint32_t via_h_cost) {
    memset(c, 0, sizeof(*c));
    c->g = g;
    c->e = e;
    c->src = net->src;
    c->dst = net->dst;
    c->win = win;
    c->plane = g->w * g->h;
    c->n = c->plane * g->layers;
    c->pads = cellset_make(net->pads, net->n_pads);
    c->via_pads = cellset_make(net->via_pads, net->n_via_pads);
    c->use_h = use_h;
    c->via_h_cost = via_h_cost;
    if (use_h) {
        c->xp = (uint64_t *)calloc(g->w + 1, sizeof(uint64_t));
        c->yp = (uint64_t *)calloc(g->h + 1, sizeof(uint64_t));
        for (uint32_t k = 0; k + 1 < g->w; ++k) c->xp[k + 1] = c->xp[k] + e->x_edge[k];
        for (uint32_t k = 0; k + 1 < g->h; ++k) c->yp[k + 1] = c->yp[k] + e->y_edge[k];
    }
}
static void iso_free(iso_ctx *c) {
    cellset_free(&c->pads);
    cellset_free(&c->via_pads);
    free(c->xp);
    free(c->yp);
}

/* One label-search engine for both forms.
 *   targeted = 1: astar_buf exactly (dijkstra.rs:243-401): the goal is not
 *                 expanded and the search stops past the equal-f frontier.
 *   targeted = 0: the complete field (h = 0, nothing skipped).
 * Labels are (dist, hops, pred) with the canonical update rules of
 * dijkstra.rs:298-375. */
static void iso_search(iso_ctx *c, int targeted, uint32_t *dist, uint32_t *hops, uint32_t *pred) {
    for (uint32_t i = 0; i < c->n; ++i) {
        dist[i] = ORC_MAX;
        hops[i] = ORC_MAX;
        pred[i] = NO_PRED;
    }
    if (iso_blocked(c, c->src)) return;
    dist[c->src] = 0;
    hops[c->src] = 0;
    heap hp = {0, 0, 0};
    heap_push(&hp, targeted ? iso_h(c, c->src) : 0, c->src);
    int goal_set = 0;
    uint32_t goal = 0;
    const orc_grid *g = c->g;
    uint32_t prio, u;
    while (heap_pop(&hp, &prio, &u)) {
        if (targeted && goal_set && prio > goal) break;
        uint32_t du = dist[u], hu = hops[u];
        uint32_t hh = targeted ? iso_h(c, u) : 0;
        if (sat_sub(prio, hh) > du) continue;
        if (targeted && u == c->dst) {
            goal = du;
            goal_set = 1;
            continue;
        }
        uint32_t layer = u / c->plane, planar = u % c->plane, x = planar % g->w;
        uint32_t nb[6];
        int isvia[6];
        int k = 0;
        if (planar >= g->w) { nb[k] = u - g->w; isvia[k++] = 0; }
        if (x > 0) { nb[k] = u - 1; isvia[k++] = 0; }
        if (x + 1 < g->w) { nb[k] = u + 1; isvia[k++] = 0; }
        if (planar + g->w < c->plane) { nb[k] = u + g->w; isvia[k++] = 0; }
        if (layer > 0) { nb[k] = u - c->plane; isvia[k++] = 1; }
        if (layer + 1 < g->layers) { nb[k] = u + c->plane; isvia[k++] = 1; }
        for (int i = 0; i < k; ++i) {
            uint32_t v = nb[i];
            if (iso_blocked(c, v)) continue;
            uint32_t step;
            if (!isvia[i]) {
                step = iso_planar_step(c, u, v);
                if (step == ORC_MAX) continue;
            } else if (!iso_via_step(c, u, v, &step)) {
                continue;
            }
            uint32_t nd = sat_add(du, step);
            uint32_t nh = sat_add(hu, 1);
            uint32_t old = dist[v];
            if (nd < old) {
                dist[v] = nd; hops[v] = nh; pred[v] = u;
                heap_push(&hp, targeted ? sat_add(nd, iso_h(c, v)) : nd, v);
            } else if (nd == old && v != c->src) {
                uint32_t oh = hops[v];
                if (nh < oh) {
                    dist[v] = nd; hops[v] = nh; pred[v] = u;
                    heap_push(&hp, targeted ? sat_add(nd, iso_h(c, v)) : nd, v);
                } else if (nh == oh && u < pred[v]) {
                    pred[v] = u;
                }
            }
        }
    }
    free(hp.a);
}

static uint32_t reverse_copy(const uint32_t *rev, uint32_t len, uint32_t *path, uint32_t cap) {
    for (uint32_t i = 0; i < len && i < cap; ++i) path[i] = rev[len - 1 - i];
    return len;
}

uint32_t orc_isolated_astar(const orc_grid *g, const orc_edges *e, const orc_net *net, orc_window win,
                            int use_heuristic, uint32_t via_h_cost, uint32_t *path, uint32_t cap,
                            uint32_t *cost_out) {
    iso_ctx c;
    iso_init(&c, g, e, net, win, use_heuristic, via_h_cost);
    uint32_t *dist = (uint32_t *)malloc(sizeof(uint32_t) * 3 * (size_t)c.n);
    uint32_t *hops = dist + c.n, *pred = hops + c.n;
    iso_search(&c, 1, dist, hops, pred);
    uint32_t len = 0;
    uint32_t total = dist[c.dst];
    if (cost_out) *cost_out = ORC_MAX;
    if (total != ORC_MAX) {
        /* reconstruction, dijkstra.rs:383-400 */
        uint32_t *rev = (uint32_t *)malloc(sizeof(uint32_t) * (c.n + 1));
        uint32_t cur = c.dst;
        rev[len++] = cur;
        int ok = 1;
        while (cur != c.src) {
            if (len > c.n) { ok = 0; break; }
            uint32_t p = pred[cur];
            if (p == NO_PRED) { ok = 0; break; }
            rev[len++] = p;
            cur = p;
        }
        if (ok) {
            reverse_copy(rev, len, path, cap);
            if (cost_out) *cost_out = total;
        } else {
            len = 0;
        }
        free(rev);
    }
    free(dist);
    iso_free(&c);
    return len;
}

void orc_isolated_field(const orc_grid *g, const orc_edges *e, const orc_net *net, orc_window win,
                        uint32_t *dist, uint32_t *hops) {
    iso_ctx c;
    iso_init(&c, g, e, net, win, 0, 0);
    uint32_t *pred = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)c.n);
    iso_search(&c, 0, dist, hops, pred);
    free(pred);
    iso_free(&c);
}

/* Backward canonical walk: candidates in ascending CellIdx (lower layer, -y, -x,
 * +x, +y, upper layer), crates/mr-metal/src/lib.rs:338-393. */
static uint32_t iso_walk(iso_ctx *c, const uint32_t *dist, const uint32_t *hops, uint32_t *path, uint32_t cap) {
    const orc_grid *g = c->g;
    if (dist[c->dst] == ORC_MAX) return 0;
    uint32_t *rev = (uint32_t *)malloc(sizeof(uint32_t) * (c->n + 1));
    uint32_t len = 0, cur = c->dst;
    rev[len++] = cur;
    while (cur != c->src) {
        uint32_t need_d = dist[cur], need_h = hops[cur];
        if (need_h == 0 || need_h == ORC_MAX) { free(rev); return 0; }
        uint32_t layer = cur / c->plane, planar = cur % c->plane, x = planar % g->w;
        uint32_t cand[6];
        int isvia[6], k = 0;
        if (layer > 0) { cand[k] = cur - c->plane; isvia[k++] = 1; }
        if (planar >= g->w) { cand[k] = cur - g->w; isvia[k++] = 0; }
        if (x > 0) { cand[k] = cur - 1; isvia[k++] = 0; }
        if (x + 1 < g->w) { cand[k] = cur + 1; isvia[k++] = 0; }
        if (planar + g->w < c->plane) { cand[k] = cur + g->w; isvia[k++] = 0; }
        if (layer + 1 < g->layers) { cand[k] = cur + c->plane; isvia[k++] = 1; }
        uint32_t next = NO_PRED;
        for (int i = 0; i < k && next == NO_PRED; ++i) {
            uint32_t p = cand[i];
            if (!iso_in_window(c, p) || dist[p] == ORC_MAX) continue;
            uint32_t step;
            if (!isvia[i]) {
                step = iso_planar_step(c, p, cur);
                if (step == ORC_MAX) continue;
            } else if (!iso_via_step(c, p, cur, &step)) {
                continue;
            }
            if (sat_add(dist[p], step) == need_d && sat_add(hops[p], 1) == need_h) next = p;
        }
        if (next == NO_PRED || len > c->n) { free(rev); return 0; }
        rev[len++] = next;
        cur = next;
    }
    reverse_copy(rev, len, path, cap);
    free(rev);
    return len;
}

uint32_t orc_isolated_path_from_labels(const orc_grid *g, const orc_edges *e, const orc_net *net, orc_window win,
                                       const uint32_t *dist, const uint32_t *hops, uint32_t *path, uint32_t cap) {
    iso_ctx c;
    iso_init(&c, g, e, net, win, 0, 0);
    uint32_t len = iso_walk(&c, dist, hops, path, cap);
    iso_free(&c);
    return len;
}

static uint32_t iso_solve_one(const orc_grid *g, const orc_edges *e, const orc_net *net, orc_window win, int mode,
                              int use_h, uint32_t via_h_cost, uint32_t *path, uint32_t cap, uint32_t *cost) {
    if (mode == 0) return orc_isolated_astar(g, e, net, win, use_h, via_h_cost, path, cap, cost);
    iso_ctx c;
    iso_init(&c, g, e, net, win, 0, 0);
    uint32_t *dist = (uint32_t *)malloc(sizeof(uint32_t) * 3 * (size_t)c.n);
    uint32_t *hops = dist + c.n, *pred = hops + c.n;
    iso_search(&c, 0, dist, hops, pred);
    uint32_t len = iso_walk(&c, dist, hops, path, cap);
    *cost = len ? dist[c.dst] : ORC_MAX;
    free(dist);
    iso_free(&c);
    return len;
}

typedef struct {
    const orc_grid *g;
    const orc_edges *e;
    const orc_net *nets;
    const orc_window *windows;
    uint32_t n_nets, n;
    int retry_full, mode, use_h;
    uint32_t via_h_cost;
    uint32_t **paths;
    uint32_t *lens, *costs;
    uint32_t next; /* work counter, taken with __atomic_fetch_add */
} batch_job;

static void *batch_worker(void *arg) {
    batch_job *j = (batch_job *)arg;
    const orc_grid *g = j->g;
    orc_window full = {0, 0, g->w ? g->w - 1 : 0, g->h ? g->h - 1 : 0};
    for (;;) {
        uint32_t i = __atomic_fetch_add(&j->next, 1, __ATOMIC_RELAXED);
        if (i >= j->n_nets) break;
        uint32_t *buf = (uint32_t *)malloc(sizeof(uint32_t) * (j->n + 1));
        uint32_t cost = ORC_MAX;
        uint32_t len = iso_solve_one(g, j->e, &j->nets[i], j->windows[i], j->mode, j->use_h, j->via_h_cost, buf,
                                     j->n + 1, &cost);
        if (len == 0 && j->retry_full)
            len = iso_solve_one(g, j->e, &j->nets[i], full, j->mode, j->use_h, j->via_h_cost, buf, j->n + 1, &cost);
        j->paths[i] = buf;
        j->lens[i] = len;
        j->costs[i] = len ? cost : ORC_MAX;
    }
    return NULL;
}

int orc_isolated_batch(const orc_grid *g, const orc_edges *e, const orc_net *nets, uint32_t n_nets,
                       const orc_window *windows, int retry_full, int mode, int use_heuristic, uint32_t via_h_cost,
                       int threads, uint64_t *offsets, uint32_t *cells, uint64_t cells_cap, uint32_t *costs) {
    batch_job j;
    j.g = g;
    j.e = e;
    j.nets = nets;
    j.windows = windows;
    j.n_nets = n_nets;
    j.n = g->w * g->h * g->layers;
    j.retry_full = retry_full;
    j.mode = mode;
    j.use_h = use_heuristic;
    j.via_h_cost = via_h_cost;
    j.paths = (uint32_t **)calloc(n_nets ? n_nets : 1, sizeof(uint32_t *));
    j.lens = (uint32_t *)calloc(n_nets ? n_nets : 1, sizeof(uint32_t));
    j.costs = costs;
    j.next = 0;
    int nt = threads > 0 ? threads : (int)sysconf(_SC_NPROCESSORS_ONLN);
    if (nt < 1) nt = 1;
    if (nt > 256) nt = 256;
    pthread_t tid[256];
    int started = 0;
    for (int t = 1; t < nt; ++t)
        if (pthread_create(&tid[started], NULL, batch_worker, &j) == 0) started++;
    batch_worker(&j);
    for (int t = 0; t < started; ++t) pthread_join(tid[t], NULL);
    uint64_t off = 0;
    int rc = 0;
    for (uint32_t i = 0; i < n_nets; ++i) {
        offsets[i] = off;
        if (off + j.lens[i] > cells_cap) rc = -1;
        else memcpy(cells + off, j.paths[i], sizeof(uint32_t) * j.lens[i]);
        off += j.lens[i];
        free(j.paths[i]);
    }
    offsets[n_nets] = off;
    free(j.paths);
    free(j.lens);
    return rc;
}

/* ------------------------------------------------------------------------ */
/* Planar per-cell-cost routines. */

uint32_t orc_lee_route_one(const orc_grid *g, const orc_net *net, uint32_t *path, uint32_t cap, uint32_t *cost_out) {
    /* LeeRouter: cost_fn(u,v) = board edge ? OBSTACLE : (own pad obstacle ? 1 :
     * cost[v]); blocked = board node || (obstacle && !pad); h = 0; no vias.
     * That is the isolated model with unit axis prices, no vias and the whole
     * board as the window, except that src/dst are not force-unblocked; the
     * router validated them already (lee.rs:77-92). */
    uint32_t one_w = g->w ? g->w - 1 : 0, one_h = g->h ? g->h - 1 : 0;
    uint32_t *ones = (uint32_t *)malloc(sizeof(uint32_t) * (one_w + one_h + 1));
    for (uint32_t i = 0; i < one_w + one_h + 1; ++i) ones[i] = 1;
    uint8_t *no_via = (uint8_t *)calloc(g->layers + 1, 1);
    orc_edges e = {ones, ones + one_w, ones, no_via, NULL};
    orc_window full = {0, 0, one_w, one_h};
    uint32_t len = orc_isolated_astar(g, &e, net, full, 0, 0, path, cap, cost_out);
    free(ones);
    free(no_via);
    return len;
}

void orc_bfs_distance_field(const orc_grid *g, uint32_t src, uint32_t *dist) {
    uint32_t n = g->w * g->h * g->layers;
    for (uint32_t i = 0; i < n; ++i) dist[i] = ORC_MAX;
    if (src >= n) return;
    if (is_obstacle(g, src) || board_trace_forbidden(g, src)) return;
    dist[src] = 0;
    heap hp = {0, 0, 0};
    heap_push(&hp, 0, src);
    uint32_t plane = g->w * g->h;
    uint32_t prio, u;
    while (heap_pop(&hp, &prio, &u)) {
        uint32_t du = dist[u];
        if (prio > du) continue;
        uint32_t layer = u / plane, r = u % plane, x = r % g->w, y = r / g->w;
        uint32_t nb[4];
        int k = 0;
        /* Dims::neighbors4 ascending order (core/src/lib.rs:129-146) */
        if (y > 0) nb[k++] = (layer * g->h + y - 1) * g->w + x;
        if (x > 0) nb[k++] = u - 1;
        if (x + 1 < g->w) nb[k++] = u + 1;
        if (y + 1 < g->h) nb[k++] = (layer * g->h + y + 1) * g->w + x;
        for (int i = 0; i < k; ++i) {
            uint32_t v = nb[i];
            if (is_obstacle(g, v) || board_trace_forbidden(g, v) || orc_board_planar_forbidden(g, u, v)) continue;
            uint32_t nd = sat_add(du, g->cost[v]);
            if (nd < dist[v]) {
                dist[v] = nd;
                heap_push(&hp, nd, v);
            }
        }
    }
    free(hp.a);
}

static uint32_t sweep_relax(const orc_grid *g, uint32_t prev, uint32_t n, uint32_t prev_dist) {
    if (prev_dist == ORC_MAX || is_obstacle(g, n) || board_trace_forbidden(g, n) || orc_board_planar_forbidden(g, prev, n))
        return ORC_MAX;
    return sat_add(prev_dist, g->cost[n]);
}

void orc_sweep_distance_field(const orc_grid *g, uint32_t src, uint32_t *dist) {
    uint32_t w = g->w, h = g->h, n = w * h * g->layers;
    for (uint32_t i = 0; i < n; ++i) dist[i] = ORC_MAX;
    if (n == 0 || src >= n || is_obstacle(g, src) || board_trace_forbidden(g, src)) return;
    dist[src] = 0;
    uint32_t layer = src / (w * h);
#define IDX3(x, y) ((layer * h + (y)) * w + (x))
    for (;;) {
        int changed = 0;
        for (uint32_t y = 0; y < h; ++y) {
            for (uint32_t x = 1; x < w; ++x) {
                uint32_t cur = IDX3(x, y), prev = IDX3(x - 1, y);
                uint32_t cand = sweep_relax(g, prev, cur, dist[prev]);
                if (cand < dist[cur]) { dist[cur] = cand; changed = 1; }
            }
            for (uint32_t xi = w - 1; xi-- > 0;) {
                uint32_t cur = IDX3(xi, y), prev = IDX3(xi + 1, y);
                uint32_t cand = sweep_relax(g, prev, cur, dist[prev]);
                if (cand < dist[cur]) { dist[cur] = cand; changed = 1; }
            }
        }
        for (uint32_t x = 0; x < w; ++x) {
            for (uint32_t y = 1; y < h; ++y) {
                uint32_t cur = IDX3(x, y), prev = IDX3(x, y - 1);
                uint32_t cand = sweep_relax(g, prev, cur, dist[prev]);
                if (cand < dist[cur]) { dist[cur] = cand; changed = 1; }
            }
            for (uint32_t yi = h - 1; yi-- > 0;) {
                uint32_t cur = IDX3(x, yi), prev = IDX3(x, yi + 1);
                uint32_t cand = sweep_relax(g, prev, cur, dist[prev]);
                if (cand < dist[cur]) { dist[cur] = cand; changed = 1; }
            }
        }
        if (!changed) break;
    }
#undef IDX3
}

uint32_t orc_path_from_field(const orc_grid *g, const uint32_t *dist, uint32_t src, uint32_t dst, uint32_t *path,
                             uint32_t cap) {
    uint32_t n = g->w * g->h * g->layers, plane = g->w * g->h;
    if (src >= n || dst >= n || is_obstacle(g, src) || is_obstacle(g, dst) || board_trace_forbidden(g, src) ||
        board_trace_forbidden(g, dst))
        return 0;
    if (dist[dst] == ORC_MAX) return 0;
    uint32_t *hops = (uint32_t *)malloc(sizeof(uint32_t) * n);
    uint32_t *queue = (uint32_t *)malloc(sizeof(uint32_t) * (n + 1));
    for (uint32_t i = 0; i < n; ++i) hops[i] = ORC_MAX;
    size_t qh = 0, qt = 0;
    hops[src] = 0;
    queue[qt++] = src;
    while (qh < qt) {
        uint32_t u = queue[qh++];
        uint32_t hu = hops[u], du = dist[u];
        if (du == ORC_MAX) continue;
        uint32_t layer = u / plane, r = u % plane, x = r % g->w, y = r / g->w;
        uint32_t nb[4];
        int k = 0;
        if (y > 0) nb[k++] = (layer * g->h + y - 1) * g->w + x;
        if (x > 0) nb[k++] = u - 1;
        if (x + 1 < g->w) nb[k++] = u + 1;
        if (y + 1 < g->h) nb[k++] = (layer * g->h + y + 1) * g->w + x;
        for (int i = 0; i < k; ++i) {
            uint32_t v = nb[i];
            if (is_obstacle(g, v) || board_trace_forbidden(g, v) || orc_board_planar_forbidden(g, u, v) ||
                sat_add(du, g->cost[v]) != dist[v] || hops[v] != ORC_MAX)
                continue;
            hops[v] = sat_add(hu, 1);
            queue[qt++] = v;
        }
    }
    uint32_t len = 0;
    if (hops[dst] != ORC_MAX) {
        uint32_t cur = dst;
        queue[len++] = cur;
        int ok = 1;
        while (cur != src) {
            uint32_t need = dist[cur], step = g->cost[cur];
            if (hops[cur] == 0) { ok = 0; break; }
            uint32_t need_h = hops[cur] - 1;
            uint32_t layer = cur / plane, r = cur % plane, x = r % g->w, y = r / g->w;
            uint32_t nb[4];
            int k = 0;
            if (y > 0) nb[k++] = (layer * g->h + y - 1) * g->w + x;
            if (x > 0) nb[k++] = cur - 1;
            if (x + 1 < g->w) nb[k++] = cur + 1;
            if (y + 1 < g->h) nb[k++] = (layer * g->h + y + 1) * g->w + x;
            uint32_t next = NO_PRED;
            for (int i = 0; i < k; ++i) {
                uint32_t p = nb[i];
                if (dist[p] != ORC_MAX && !orc_board_planar_forbidden(g, p, cur) && sat_add(dist[p], step) == need &&
                    hops[p] == need_h) {
                    next = p;
                    break;
                }
            }
            if (next == NO_PRED) { ok = 0; break; }
            queue[len++] = next;
            cur = next;
        }
        if (ok) {
            for (uint32_t i = 0; i < len && i < cap; ++i) path[i] = queue[len - 1 - i];
        } else {
            len = 0;
        }
    }
    free(hops);
    free(queue);
    return len;
}

/* ------------------------------------------------------------------------ */

int orc_provider_path_is_valid(const orc_grid *g, const uint8_t *via_allowed, const orc_net *net, const uint32_t *path,
                               uint32_t len) {
    uint32_t n = g->w * g->h * g->layers, plane = g->w * g->h;
    if (len == 0 || len > n || path[0] != net->src || path[len - 1] != net->dst) return 0;
    cellset pads = cellset_make(net->pads, net->n_pads);
    cellset vpads = cellset_make(net->via_pads, net->n_via_pads);
    cellset seen = cellset_make(path, len);
    int ok = seen.n == len;
    for (uint32_t i = 0; ok && i < len; ++i) {
        uint32_t c = path[i];
        if (c >= n || board_trace_forbidden(g, c) || (is_obstacle(g, c) && !cellset_has(&pads, c))) ok = 0;
    }
    for (uint32_t i = 0; ok && i + 1 < len; ++i) {
        uint32_t a = path[i], b = path[i + 1];
        uint32_t al = a / plane, bl = b / plane, ar = a % plane, br = b % plane;
        uint32_t ax = ar % g->w, ay = ar / g->w, bx = br % g->w, by = br / g->w;
        if (al == bl) {
            int adj = ((ax + 1 == bx || bx + 1 == ax) && ay == by) || ((ay + 1 == by || by + 1 == ay) && ax == bx);
            ok = adj && !orc_board_planar_forbidden(g, a, b);
        } else {
            uint32_t lo = al < bl ? al : bl, hi = al < bl ? bl : al;
            int legal = (hi == lo + 1) && hi < g->layers && via_allowed && via_allowed[lo];
            ok = ax == bx && ay == by && legal && !board_via_forbidden(g, a) && !board_via_forbidden(g, b) &&
                 (!static_via_forbidden(g, a) || cellset_has(&vpads, a)) &&
                 (!static_via_forbidden(g, b) || cellset_has(&vpads, b));
        }
    }
    cellset_free(&pads);
    cellset_free(&vpads);
    cellset_free(&seen);
    return ok;
}
