/*
 * oracle.c — CPU oracle for incremental subgraph matching under edge-update batches.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker of the B200 engine: only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.  The engine never calls it.
 *
 * It restates the semantics the reference GCSM-BU counts, independently of any GPU design:
 *  - graph/graph.cpp:191-269, 359-468: labelled, undirected query and data graphs; an edge
 *    (u, v, l) of the data graph matches query edge (a, b, l) in both orientations.
 *  - technique_permutation.h:224 "Num Positive Matches": embeddings are injective maps f with
 *    equal vertex labels and every query edge present with its label (non-induced);
 *    automorphic images are distinct embeddings (no symmetry breaking:
 *    graph/match_gpu.cu:278-286 sets C_EQUIV_EDGE_COUNT to 1).
 *  - technique_permutation.h:125-212: per batch, query edges are processed in qe_list_ order
 *    (graph.cpp:332-347) and query edge i counts the embeddings whose query edge i maps to a
 *    batch edge while every query edge after i maps to an edge that was already present.
 *    The sum over i is |M(G')| - |M(G)| for an insert-only batch.
 * Deletions (no reference counterpart) use the mirror rule on the graph before the batch:
 * a batch means G' = (G \ Del) U Ins; D = G \ G', I = G' \ G; the negative count is the
 * number of embeddings of G that use an edge of D, the positive count the number of
 * embeddings of G' that use an edge of I.
 *
 * Search: backtracking from every batch edge in both orientations, vertices in BFS order
 * from the updated edge (plan.cpp:1548-1577), candidates scanned from the first backward
 * neighbour, the other backward edges checked by binary search.  Work items (query edge,
 * batch edge, orientation) are shared by POSIX threads through an atomic counter.
 */
#define _GNU_SOURCE
#include <pthread.h>
#include <stdatomic.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#define MAXQV 16
#define MAXQE 42

typedef struct {
    uint32_t v, l;
} Nbr;

typedef struct {
    Nbr *a;
    uint32_t n, cap;
} Adj;

typedef struct {
    uint32_t x, y, l; /* x < y */
} EKey;

typedef struct {
    /* query */
    uint32_t qn, qm;
    uint32_t qlab[MAXQV];
    int qidx[MAXQV][MAXQV];      /* qe_list index of (u, uu), -1 if not adjacent */
    uint32_t qel[MAXQV][MAXQV];  /* edge label */
    uint32_t qe_a[MAXQE], qe_b[MAXQE], qe_l[MAXQE];
    /* data graph */
    uint32_t nv;
    uint32_t *vlab;
    Adj *adj;
    /* last batch results */
    uint64_t pos, neg;
    uint64_t per_qe[2][MAXQE];
    uint32_t *rows[2];
    uint64_t nrows[2];
    uint64_t b_scan, b_probe; /* adjacency entries scanned, membership probes */
} Oracle;

static int nbr_cmp(const Nbr *a, uint32_t v, uint32_t l) {
    if (a->v != v) return a->v < v ? -1 : 1;
    if (a->l != l) return a->l < l ? -1 : 1;
    return 0;
}

/* First index with (v, l) >= key. */
static uint32_t adj_lb(const Adj *A, uint32_t v, uint32_t l) {
    uint32_t lo = 0, hi = A->n;
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (nbr_cmp(&A->a[mid], v, l) < 0) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

static int has_edge(const Oracle *o, uint32_t x, uint32_t y, uint32_t l) {
    if (x >= o->nv || y >= o->nv) return 0;
    const Adj *A = &o->adj[x];
    uint32_t i = adj_lb(A, y, l);
    return i < A->n && A->a[i].v == y && A->a[i].l == l;
}

static int adj_insert(Adj *A, uint32_t v, uint32_t l) {
    uint32_t i = adj_lb(A, v, l);
    if (i < A->n && A->a[i].v == v && A->a[i].l == l) return 0;
    if (A->n == A->cap) {
        uint32_t nc = A->cap ? A->cap * 2 : 4;
        Nbr *na = (Nbr *)realloc(A->a, sizeof(Nbr) * nc);
        if (!na) return -1;
        A->a = na;
        A->cap = nc;
    }
    memmove(A->a + i + 1, A->a + i, sizeof(Nbr) * (A->n - i));
    A->a[i].v = v;
    A->a[i].l = l;
    A->n++;
    return 1;
}

static int adj_remove(Adj *A, uint32_t v, uint32_t l) {
    uint32_t i = adj_lb(A, v, l);
    if (!(i < A->n && A->a[i].v == v && A->a[i].l == l)) return 0;
    memmove(A->a + i, A->a + i + 1, sizeof(Nbr) * (A->n - i - 1));
    A->n--;
    return 1;
}

static int nbr_sort_cmp(const void *pa, const void *pb) {
    const Nbr *a = (const Nbr *)pa, *b = (const Nbr *)pb;
    if (a->v != b->v) return a->v < b->v ? -1 : 1;
    if (a->l != b->l) return a->l < b->l ? -1 : 1;
    return 0;
}

static int ekey_cmp(const void *pa, const void *pb) {
    const EKey *a = (const EKey *)pa, *b = (const EKey *)pb;
    if (a->x != b->x) return a->x < b->x ? -1 : 1;
    if (a->y != b->y) return a->y < b->y ? -1 : 1;
    if (a->l != b->l) return a->l < b->l ? -1 : 1;
    return 0;
}

static EKey mk(uint32_t x, uint32_t y, uint32_t l) {
    EKey k;
    k.x = x < y ? x : y;
    k.y = x < y ? y : x;
    k.l = l;
    return k;
}

static int in_set(const EKey *s, uint64_t n, uint32_t x, uint32_t y, uint32_t l) {
    EKey k = mk(x, y, l);
    uint64_t lo = 0, hi = n;
    while (lo < hi) {
        uint64_t mid = (lo + hi) >> 1;
        int c = ekey_cmp(&s[mid], &k);
        if (c < 0) lo = mid + 1;
        else hi = mid;
    }
    return lo < n && ekey_cmp(&s[lo], &k) == 0;
}

void *oracle_create(uint32_t qn, const uint32_t *qvl, uint32_t qm, const uint32_t *qs, const uint32_t *qd,
                    const uint32_t *ql, uint32_t nv, const uint32_t *vl, uint64_t ne, const uint32_t *es,
                    const uint32_t *ed, const uint32_t *el) {
    if (qn < 2 || qn > MAXQV || qm == 0 || qm > MAXQE) return NULL;
    Oracle *o = (Oracle *)calloc(1, sizeof(Oracle));
    if (!o) return NULL;
    o->qn = qn;
    o->qm = qm;
    memcpy(o->qlab, qvl, sizeof(uint32_t) * qn);
    for (uint32_t a = 0; a < MAXQV; a++)
        for (uint32_t b = 0; b < MAXQV; b++) o->qidx[a][b] = -1;
    int adjq[MAXQV][MAXQV];
    memset(adjq, 0, sizeof adjq);
    for (uint32_t e = 0; e < qm; e++) {
        adjq[qs[e]][qd[e]] = adjq[qd[e]][qs[e]] = 1;
        o->qel[qs[e]][qd[e]] = o->qel[qd[e]][qs[e]] = ql[e];
    }
    /* qe_list_ order: u ascending, then neighbour ascending, u < uu (graph.cpp:332-347). */
    uint32_t k = 0;
    for (uint32_t u = 0; u < qn; u++)
        for (uint32_t uu = u + 1; uu < qn; uu++)
            if (adjq[u][uu]) {
                o->qidx[u][uu] = o->qidx[uu][u] = (int)k;
                o->qe_a[k] = u;
                o->qe_b[k] = uu;
                o->qe_l[k] = o->qel[u][uu];
                k++;
            }
    o->nv = nv;
    o->vlab = (uint32_t *)malloc(sizeof(uint32_t) * (nv ? nv : 1));
    o->adj = (Adj *)calloc(nv ? nv : 1, sizeof(Adj));
    if (!o->vlab || !o->adj) return NULL;
    memcpy(o->vlab, vl, sizeof(uint32_t) * nv);
    /* Bulk build: count, fill, then sort and deduplicate each list. */
    uint32_t *deg = (uint32_t *)calloc(nv ? nv : 1, sizeof(uint32_t));
    if (!deg) return NULL;
    for (uint64_t e = 0; e < ne; e++) {
        uint32_t x = es[e], y = ed[e];
        if (x >= nv || y >= nv || x == y) continue;
        deg[x]++;
        deg[y]++;
    }
    for (uint32_t v = 0; v < nv; v++) {
        o->adj[v].cap = deg[v] ? deg[v] : 0;
        o->adj[v].a = deg[v] ? (Nbr *)malloc(sizeof(Nbr) * deg[v]) : NULL;
        if (deg[v] && !o->adj[v].a) return NULL;
    }
    for (uint64_t e = 0; e < ne; e++) {
        uint32_t x = es[e], y = ed[e];
        if (x >= nv || y >= nv || x == y) continue;
        Adj *A = &o->adj[x], *B = &o->adj[y];
        A->a[A->n].v = y;
        A->a[A->n++].l = el[e];
        B->a[B->n].v = x;
        B->a[B->n++].l = el[e];
    }
    for (uint32_t v = 0; v < nv; v++) {
        Adj *A = &o->adj[v];
        if (A->n < 2) continue;
        qsort(A->a, A->n, sizeof(Nbr), nbr_sort_cmp);
        uint32_t w = 1;
        for (uint32_t i = 1; i < A->n; i++)
            if (A->a[i].v != A->a[w - 1].v || A->a[i].l != A->a[w - 1].l) A->a[w++] = A->a[i];
        A->n = w;
    }
    free(deg);
    return o;
}

void oracle_destroy(void *h) {
    Oracle *o = (Oracle *)h;
    if (!o) return;
    for (uint32_t v = 0; v < o->nv; v++) free(o->adj[v].a);
    free(o->adj);
    free(o->vlab);
    free(o->rows[0]);
    free(o->rows[1]);
    free(o);
}

/* ---- seeded enumeration ---- */

typedef struct {
    uint32_t n;
    uint8_t order[MAXQV];
    uint8_t nbn[MAXQV];
    uint8_t bn[MAXQV][MAXQV];  /* depths of backward neighbours */
} Order;

static void bfs_order(const Oracle *o, uint32_t a, uint32_t b, Order *ord) {
    int vis[MAXQV] = {0};
    uint32_t n = 0;
    ord->order[n++] = (uint8_t)a;
    ord->order[n++] = (uint8_t)b;
    vis[a] = vis[b] = 1;
    uint32_t head = 0;
    while (head < n) {
        uint32_t v = ord->order[head++];
        for (uint32_t w = 0; w < o->qn; w++)
            if (!vis[w] && o->qidx[v][w] >= 0) {
                vis[w] = 1;
                ord->order[n++] = (uint8_t)w;
            }
    }
    ord->n = n;
    for (uint32_t d = 0; d < n; d++) {
        ord->nbn[d] = 0;
        for (uint32_t k = 0; k < d; k++)
            if (o->qidx[ord->order[k]][ord->order[d]] >= 0) ord->bn[d][ord->nbn[d]++] = (uint8_t)k;
    }
}

typedef struct {
    const Oracle *o;
    const EKey *newset;
    uint64_t nnew;
    Order ord[MAXQE];
    atomic_ulong next;
    uint64_t nitems; /* qm * nnew * 2 */
    uint64_t stride; /* items are visited in the order (k * stride) mod nitems */
    int want_rows;
    double deadline; /* CLOCK_MONOTONIC seconds; 0 = none */
    atomic_ulong done;
} Job;

static double now_s(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

static uint64_t gcd64(uint64_t a, uint64_t b) {
    while (b) {
        uint64_t t = a % b;
        a = b;
        b = t;
    }
    return a;
}

typedef struct {
    Job *job;
    uint64_t per_qe[MAXQE];
    uint32_t *rows;
    uint64_t nrows, cap;
    uint64_t scan, probe;
    int oom;
    int stop; /* deadline passed inside an item */
} Worker;

static void emit_row(Worker *w, const Order *ord, const uint32_t *f) {
    const uint32_t n = ord->n;
    if (w->nrows == w->cap) {
        uint64_t nc = w->cap ? w->cap * 2 : 1024;
        uint32_t *nr = (uint32_t *)realloc(w->rows, sizeof(uint32_t) * n * nc);
        if (!nr) {
            w->oom = 1;
            return;
        }
        w->rows = nr;
        w->cap = nc;
    }
    uint32_t *row = w->rows + w->nrows * n;
    for (uint32_t d = 0; d < n; d++) row[ord->order[d]] = f[d];
    w->nrows++;
}

static void extend(Worker *w, uint32_t qe, const Order *ord, uint32_t d, uint32_t *f) {
    const Oracle *o = w->job->o;
    if (d == ord->n) {
        w->per_qe[qe]++;
        if (w->job->want_rows) emit_row(w, ord, f);
        return;
    }
    const uint32_t u = ord->order[d];
    /* Scan the smallest backward-neighbour list, probe the others. */
    uint32_t pk = 0;
    for (uint32_t b = 1; b < ord->nbn[d]; b++)
        if (o->adj[f[ord->bn[d][b]]].n < o->adj[f[ord->bn[d][pk]]].n) pk = b;
    const uint32_t p = ord->bn[d][pk];
    const uint32_t pu = ord->order[p];
    const uint32_t l0 = o->qel[pu][u];
    const int old0 = o->qidx[pu][u] > (int)qe;
    const Adj *A = &o->adj[f[p]];
    for (uint32_t i = 0; i < A->n && !w->stop; i++) {
        const uint32_t c = A->a[i].v;
        if ((++w->scan & 4095u) == 0 && w->job->deadline > 0 && now_s() > w->job->deadline) w->stop = 1;
        if (A->a[i].l != l0 || o->vlab[c] != o->qlab[u]) continue;
        int ok = 1;
        for (uint32_t k = 0; k < d && ok; k++) ok = f[k] != c;
        if (!ok) continue;
        if (old0 && in_set(w->job->newset, w->job->nnew, f[p], c, l0)) continue;
        for (uint32_t b = 0; b < ord->nbn[d] && ok; b++) {
            if (b == pk) continue;
            const uint32_t bd = ord->bn[d][b];
            const uint32_t bu = ord->order[bd];
            const uint32_t lb = o->qel[bu][u];
            w->probe++;
            ok = has_edge(o, f[bd], c, lb);
            if (ok && o->qidx[bu][u] > (int)qe) ok = !in_set(w->job->newset, w->job->nnew, f[bd], c, lb);
        }
        if (!ok) continue;
        f[d] = c;
        extend(w, qe, ord, d + 1, f);
    }
}

static void *worker_main(void *arg) {
    Worker *w = (Worker *)arg;
    Job *job = w->job;
    const Oracle *o = job->o;
    uint32_t f[MAXQV];
    for (;;) {
        uint64_t k = atomic_fetch_add(&job->next, 1);
        if (k >= job->nitems || w->stop) break;
        if (job->deadline > 0 && now_s() > job->deadline) break;
        atomic_fetch_add(&job->done, 1);
        const uint64_t it = (k * job->stride) % job->nitems;
        const uint32_t qe = (uint32_t)(it / (job->nnew * 2));
        const uint64_t rem = it % (job->nnew * 2);
        const EKey *e = &job->newset[rem / 2];
        if (e->l != o->qe_l[qe]) continue;
        const uint32_t x = (rem & 1) ? e->y : e->x, y = (rem & 1) ? e->x : e->y;
        const Order *ord = &job->ord[qe];
        /* order[0], order[1] are the endpoints qe_a, qe_b of query edge qe. */
        if (o->vlab[x] != o->qlab[ord->order[0]] || o->vlab[y] != o->qlab[ord->order[1]]) continue;
        f[0] = x;
        f[1] = y;
        extend(w, qe, ord, 2, f);
    }
    return NULL;
}

static uint32_t g_row_n;
static int row_cmp(const void *a, const void *b) {
    const uint32_t *x = (const uint32_t *)a, *y = (const uint32_t *)b;
    for (uint32_t i = 0; i < g_row_n; i++)
        if (x[i] != y[i]) return x[i] < y[i] ? -1 : 1;
    return 0;
}

/* Counts embeddings of the current graph that use >= 1 edge of `newset` (sorted, unique). */
static int delta(Oracle *o, const EKey *newset, uint64_t nnew, int nthreads, int want_rows, uint64_t *per_qe,
                 uint32_t **rows_out, uint64_t *nrows_out, double deadline, uint64_t *items) {
    Job job;
    memset(&job, 0, sizeof job);
    job.o = o;
    job.newset = newset;
    job.nnew = nnew;
    job.want_rows = want_rows;
    job.nitems = (uint64_t)o->qm * nnew * 2;
    job.deadline = deadline;
    job.stride = 1;
    if (deadline > 0 && job.nitems > 1) {
        /* Sampling: visit items in a scattered order so a deadline cuts an unbiased subset. */
        uint64_t st = 2654435761ull % job.nitems;
        while (st < 2 || gcd64(st, job.nitems) != 1) st++;
        job.stride = st;
    }
    atomic_init(&job.next, 0);
    atomic_init(&job.done, 0);
    for (uint32_t i = 0; i < o->qm; i++) bfs_order(o, o->qe_a[i], o->qe_b[i], &job.ord[i]);
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    Worker *ws = (Worker *)calloc((size_t)nthreads, sizeof(Worker));
    pthread_t *th = (pthread_t *)calloc((size_t)nthreads, sizeof(pthread_t));
    if (!ws || !th) return -1;
    for (int t = 0; t < nthreads; t++) {
        ws[t].job = &job;
        if (nnew && t > 0) pthread_create(&th[t], NULL, worker_main, &ws[t]);
    }
    if (nnew) worker_main(&ws[0]);
    for (int t = 1; t < nthreads; t++)
        if (nnew) pthread_join(th[t], NULL);
    int rc = 0;
    uint64_t total_rows = 0;
    for (int t = 0; t < nthreads; t++) {
        for (uint32_t i = 0; i < o->qm; i++) per_qe[i] += ws[t].per_qe[i];
        total_rows += ws[t].nrows;
        o->b_scan += ws[t].scan;
        o->b_probe += ws[t].probe;
        if (ws[t].oom) rc = -1;
    }
    if (want_rows) {
        uint32_t *all = (uint32_t *)malloc(sizeof(uint32_t) * o->qn * (total_rows ? total_rows : 1));
        if (!all) rc = -1;
        uint64_t k = 0;
        for (int t = 0; t < nthreads && all; t++) {
            memcpy(all + k * o->qn, ws[t].rows, sizeof(uint32_t) * o->qn * ws[t].nrows);
            k += ws[t].nrows;
        }
        if (all) {
            g_row_n = o->qn;
            qsort(all, total_rows, sizeof(uint32_t) * o->qn, row_cmp);
        }
        *rows_out = all;
        *nrows_out = total_rows;
    }
    if (items) *items += atomic_load(&job.done);
    for (int t = 0; t < nthreads; t++) free(ws[t].rows);
    free(ws);
    free(th);
    return rc;
}

/*
 * Applies one batch; fills out[0] = positive, out[1] = negative and per_qe[0..qm) positive,
 * per_qe[qm..2qm) negative counts per query edge (qe_list_ order).  Returns 0 on success.
 */
static int apply_impl(void *h, uint64_t nb, const uint32_t *bs, const uint32_t *bd, const uint32_t *bl,
                      const uint8_t *bdel, int nthreads, int want_rows, uint64_t *out, uint64_t *per_qe,
                      double max_seconds, uint64_t *items) {
    Oracle *o = (Oracle *)h;
    const double deadline = max_seconds > 0 ? now_s() + max_seconds : 0.0;
    if (!o) return -1;
    /* Net effect of the batch: an insertion wins over a deletion of the same edge. */
    EKey *ins = (EKey *)malloc(sizeof(EKey) * (nb + 1)), *del = (EKey *)malloc(sizeof(EKey) * (nb + 1));
    if (!ins || !del) return -1;
    uint64_t ni = 0, nd = 0;
    for (uint64_t i = 0; i < nb; i++) {
        const uint32_t x = bs[i], y = bd[i];
        if (x >= o->nv || y >= o->nv || x == y) continue;
        if (bdel && bdel[i]) del[nd++] = mk(x, y, bl[i]);
        else ins[ni++] = mk(x, y, bl[i]);
    }
    qsort(ins, ni, sizeof(EKey), ekey_cmp);
    qsort(del, nd, sizeof(EKey), ekey_cmp);
    uint64_t w = 0;
    for (uint64_t i = 0; i < ni; i++)
        if (i == 0 || ekey_cmp(&ins[i], &ins[i - 1]) != 0) ins[w++] = ins[i];
    ni = w;
    w = 0;
    for (uint64_t i = 0; i < nd; i++)
        if ((i == 0 || ekey_cmp(&del[i], &del[i - 1]) != 0) && !in_set(ins, ni, del[i].x, del[i].y, del[i].l))
            del[w++] = del[i];
    nd = w;
    /* D = deletions present in G; I = insertions absent from G. */
    w = 0;
    for (uint64_t i = 0; i < nd; i++)
        if (has_edge(o, del[i].x, del[i].y, del[i].l)) del[w++] = del[i];
    nd = w;
    w = 0;
    for (uint64_t i = 0; i < ni; i++)
        if (!has_edge(o, ins[i].x, ins[i].y, ins[i].l)) ins[w++] = ins[i];
    ni = w;

    memset(o->per_qe, 0, sizeof o->per_qe);
    free(o->rows[0]);
    free(o->rows[1]);
    o->rows[0] = o->rows[1] = NULL;
    o->nrows[0] = o->nrows[1] = 0;
    o->b_scan = o->b_probe = 0;
    int rc = 0;
    /* Negative: on G, with D as the batch edges. */
    rc |= delta(o, del, nd, nthreads, want_rows, o->per_qe[1], &o->rows[1], &o->nrows[1], deadline, items);
    for (uint64_t i = 0; i < nd; i++) {
        adj_remove(&o->adj[del[i].x], del[i].y, del[i].l);
        adj_remove(&o->adj[del[i].y], del[i].x, del[i].l);
    }
    for (uint64_t i = 0; i < ni; i++) {
        adj_insert(&o->adj[ins[i].x], ins[i].y, ins[i].l);
        adj_insert(&o->adj[ins[i].y], ins[i].x, ins[i].l);
    }
    /* Positive: on G', with I as the batch edges. */
    rc |= delta(o, ins, ni, nthreads, want_rows, o->per_qe[0], &o->rows[0], &o->nrows[0], deadline, items);
    o->pos = o->neg = 0;
    for (uint32_t i = 0; i < o->qm; i++) {
        o->pos += o->per_qe[0][i];
        o->neg += o->per_qe[1][i];
    }
    if (out) {
        out[0] = o->pos;
        out[1] = o->neg;
        out[2] = ni;
        out[3] = nd;
    }
    if (per_qe)
        for (uint32_t i = 0; i < o->qm; i++) {
            per_qe[i] = o->per_qe[0][i];
            per_qe[o->qm + i] = o->per_qe[1][i];
        }
    free(ins);
    free(del);
    return rc;
}

int oracle_apply(void *h, uint64_t nb, const uint32_t *bs, const uint32_t *bd, const uint32_t *bl, const uint8_t *bdel,
                 int nthreads, int want_rows, uint64_t *out, uint64_t *per_qe) {
    return apply_impl(h, nb, bs, bd, bl, bdel, nthreads, want_rows, out, per_qe, 0.0, NULL);
}

/*
 * Throughput sample: applies the batch to the graph like oracle_apply but stops counting
 * once `max_seconds` have passed (the counts then cover a scattered subset of the work
 * items); *items receives the number of (query edge, batch edge, orientation) items done.
 */
int oracle_apply_sample(void *h, uint64_t nb, const uint32_t *bs, const uint32_t *bd, const uint32_t *bl,
                        const uint8_t *bdel, int nthreads, double max_seconds, uint64_t *out, uint64_t *items) {
    uint64_t per[2 * MAXQE];
    *items = 0;
    return apply_impl(h, nb, bs, bd, bl, bdel, nthreads, 0, out, per, max_seconds, items);
}

/* Copies the sorted rows of the last batch (sign > 0 positive, < 0 negative); returns the count. */
uint64_t oracle_rows(void *h, int sign, uint32_t *buf, uint64_t cap_rows) {
    Oracle *o = (Oracle *)h;
    const int s = sign >= 0 ? 0 : 1;
    const uint64_t n = o->nrows[s];
    if (buf && o->rows[s]) memcpy(buf, o->rows[s], sizeof(uint32_t) * o->qn * (n < cap_rows ? n : cap_rows));
    return n;
}

/* Adjacency entries scanned and membership probes of the last batch (canonical work counts). */
void oracle_work(void *h, uint64_t *scan, uint64_t *probe) {
    Oracle *o = (Oracle *)h;
    *scan = o->b_scan;
    *probe = o->b_probe;
}

/* |M(G)|: every embedding of the current graph (small graphs only; single thread). */
static void full_extend(const Oracle *o, const Order *ord, uint32_t d, uint32_t *f, uint64_t *cnt) {
    if (d == ord->n) {
        (*cnt)++;
        return;
    }
    const uint32_t u = ord->order[d];
    const uint32_t p = ord->bn[d][0];
    const uint32_t l0 = o->qel[ord->order[p]][u];
    const Adj *A = &o->adj[f[p]];
    for (uint32_t i = 0; i < A->n; i++) {
        const uint32_t c = A->a[i].v;
        if (A->a[i].l != l0 || o->vlab[c] != o->qlab[u]) continue;
        int ok = 1;
        for (uint32_t k = 0; k < d && ok; k++) ok = f[k] != c;
        for (uint32_t b = 1; b < ord->nbn[d] && ok; b++) {
            const uint32_t bd = ord->bn[d][b];
            ok = has_edge(o, f[bd], c, o->qel[ord->order[bd]][u]);
        }
        if (!ok) continue;
        f[d] = c;
        full_extend(o, ord, d + 1, f, cnt);
    }
}

uint64_t oracle_count_all(void *h) {
    Oracle *o = (Oracle *)h;
    Order ord;
    bfs_order(o, o->qe_a[0], o->qe_b[0], &ord);
    uint64_t cnt = 0;
    uint32_t f[MAXQV];
    for (uint32_t x = 0; x < o->nv; x++) {
        if (o->vlab[x] != o->qlab[ord.order[0]]) continue;
        const Adj *A = &o->adj[x];
        for (uint32_t i = 0; i < A->n; i++) {
            const uint32_t y = A->a[i].v;
            if (A->a[i].l != o->qe_l[0] || o->vlab[y] != o->qlab[ord.order[1]]) continue;
            f[0] = x;
            f[1] = y;
            full_extend(o, &ord, 2, f, &cnt);
        }
    }
    return cnt;
}
