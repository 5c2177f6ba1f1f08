/* Plain-C restatement of the reference's SVG construction (the ICH window
 * propagation of ICHDevice.cu and the per-source loop of SVG.cu) and of its
 * host graph search.  TEST ORACLE ONLY: tests/, the smoke check and
 * bench.py's CPU-baseline leg use it to check the CUDA product.
 *
 * Each routine cites the reference lines it restates.  The arithmetic is the
 * reference's, operation for operation, compiled with -ffp-contract=off so no
 * multiply-add is fused: results are bit-identical to the reference compiled
 * the same way (checked in tests/test_oracle.py).
 *
 * Deliberate deviations, all outside the reference's defined behaviour:
 *   - boundary half-edges get twin -1 (the reference leaves 0, Mesh.cu:62);
 *   - nextToSrcX/nextToDstX are 0.0 when the reference leaves them unset;
 *   - a watchdog caps every loop (flags bit1) where the reference could spin.
 */
#define _GNU_SOURCE
#include "svg_oracle.h"

#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>

#define REF_PI 3.141592653589793238     /* Geometry.cuh:18 */
#define RELATIVE_ERROR 1e-8             /* ICHDevice.cuh:10 */
#define WATCHDOG (1LL << 26)      /* ICH loop steps per source */
#define FAN_GUARD (1LL << 20)     /* fan walk / vertex ring steps */

/* ------------------------------------------------------------------ mesh */
struct om_mesh {
    int nv, nf, ne;
    double* pos;     /* nv*3 */
    int32_t* faces;  /* nf*3 */
    int32_t* v0;     /* edges[e].verts[0] */
    int32_t* v1;     /* edges[e].verts[1] */
    int32_t* twin, *next, *prev, *face;
    double* len;
    double* angle;
    int32_t* first;
};

typedef struct { int64_t key; int val; } kv_t;

static uint64_t mix64(uint64_t x) {
    x ^= x >> 33; x *= 0xff51afd7ed558ccdULL; x ^= x >> 33; x *= 0xc4ceb9fe1a85ec53ULL; x ^= x >> 33;
    return x;
}

/* Mesh.cu:62-123: half-edge 3f+j runs verts[j] -> verts[(j+1)%3]; twins are
 * paired through a map keyed by the sorted vertex pair (the first half-edge
 * seen for a pair is the map entry; each later one pairs with it); the
 * vertex angle is the sum, in half-edge order, of the corner angle at
 * verts[0]; firstEdge is the last half-edge leaving the vertex. */
int om_mesh_create(int nv, const double* pos, int nf, const int32_t* faces, om_mesh** out) {
    om_mesh* m = (om_mesh*)calloc(1, sizeof(om_mesh));
    if (!m) return 1;
    int ne = 3 * nf;
    m->nv = nv; m->nf = nf; m->ne = ne;
    m->pos = (double*)malloc(sizeof(double) * 3 * (size_t)(nv > 0 ? nv : 1));
    m->faces = (int32_t*)malloc(sizeof(int32_t) * 3 * (size_t)(nf > 0 ? nf : 1));
    size_t E = (size_t)(ne > 0 ? ne : 1);
    m->v0 = (int32_t*)malloc(4 * E); m->v1 = (int32_t*)malloc(4 * E);
    m->twin = (int32_t*)malloc(4 * E); m->next = (int32_t*)malloc(4 * E);
    m->prev = (int32_t*)malloc(4 * E); m->face = (int32_t*)malloc(4 * E);
    m->len = (double*)malloc(8 * E);
    m->angle = (double*)calloc((size_t)(nv > 0 ? nv : 1), 8);
    m->first = (int32_t*)malloc(4 * (size_t)(nv > 0 ? nv : 1));
    memcpy(m->pos, pos, sizeof(double) * 3 * (size_t)nv);
    memcpy(m->faces, faces, sizeof(int32_t) * 3 * (size_t)nf);
    for (int v = 0; v < nv; ++v) m->first[v] = -1;

    size_t cap = 16;
    while (cap < 2 * E) cap <<= 1;
    kv_t* tab = (kv_t*)malloc(sizeof(kv_t) * cap);
    for (size_t i = 0; i < cap; ++i) tab[i].key = -1;
    for (int f = 0; f < nf; ++f) {
        for (int j = 0; j < 3; ++j) {
            int e = 3 * f + j;
            int a = faces[3 * f + j], b = faces[3 * f + (j + 1) % 3];
            m->v0[e] = a; m->v1[e] = b;
            double dx = pos[3 * a] - pos[3 * b], dy = pos[3 * a + 1] - pos[3 * b + 1],
                   dz = pos[3 * a + 2] - pos[3 * b + 2];
            m->len[e] = sqrt(dx * dx + dy * dy + dz * dz);
            m->next[e] = 3 * f + (j + 1) % 3;
            m->prev[e] = 3 * f + (j + 2) % 3;
            m->face[e] = f;
            m->twin[e] = -1;
            int lo = a < b ? a : b, hi = a < b ? b : a;
            int64_t key = ((int64_t)lo << 32) | (uint32_t)hi;
            size_t h = mix64((uint64_t)key) & (cap - 1);
            while (tab[h].key != -1 && tab[h].key != key) h = (h + 1) & (cap - 1);
            if (tab[h].key == key) {
                m->twin[e] = tab[h].val;
                m->twin[tab[h].val] = e;
            } else {
                tab[h].key = key;
                tab[h].val = e;
            }
        }
    }
    free(tab);
    for (int i = 0; i < ne; ++i) {
        double l0 = m->len[i], l1 = m->len[m->next[i]], l2 = m->len[m->prev[i]];
        double c = (l0 * l0 + l2 * l2 - l1 * l1) / (2.0 * l0 * l2);
        if (c > 1.0) c = 1.0; else if (c < -1.0) c = -1.0;
        c = acos(c);
        m->angle[m->v0[i]] += c;
        m->first[m->v0[i]] = i;
    }
    *out = m;
    return 0;
}

void om_mesh_free(om_mesh* m) {
    if (!m) return;
    free(m->pos); free(m->faces); free(m->v0); free(m->v1); free(m->twin); free(m->next);
    free(m->prev); free(m->face); free(m->len); free(m->angle); free(m->first);
    free(m);
}

void om_mesh_counts(const om_mesh* m, int* nv, int* nf, int* ne) {
    *nv = m->nv; *nf = m->nf; *ne = m->ne;
}

void om_mesh_export(const om_mesh* m, int32_t* he_v0, int32_t* he_twin, double* he_len,
                    double* angle, int32_t* first_edge) {
    if (he_v0) memcpy(he_v0, m->v0, 4 * (size_t)m->ne);
    if (he_twin) memcpy(he_twin, m->twin, 4 * (size_t)m->ne);
    if (he_len) memcpy(he_len, m->len, 8 * (size_t)m->ne);
    if (angle) memcpy(angle, m->angle, 8 * (size_t)m->nv);
    if (first_edge) memcpy(first_edge, m->first, 4 * (size_t)m->nv);
}

/* ------------------------------------------------------------- 2D math */
typedef struct { double x, y; } vec2;
static inline vec2 mk(double x, double y) { vec2 r; r.x = x; r.y = y; return r; }
static inline vec2 sub(vec2 a, vec2 b) { return mk(a.x - b.x, a.y - b.y); }
static inline vec2 add(vec2 a, vec2 b) { return mk(a.x + b.x, a.y + b.y); }
static inline vec2 scl(double u, vec2 a) { return mk(a.x * u, a.y * u); }   /* Geometry.cu:55-60 */
static inline double dot(vec2 a, vec2 b) { return a.x * b.x + a.y * b.y; }  /* Geometry.cu:76 */
static inline double cross(vec2 a, vec2 b) { return a.x * b.y - a.y * b.x; } /* Geometry.cu:81 */
static inline double len2d(vec2 a) { return sqrt(a.x * a.x + a.y * a.y); }  /* Geometry.cuh:33 */
static inline double len3(const double* a, const double* b) {
    double dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
    return sqrt(dx * dx + dy * dy + dz * dz);
}
/* Vector2D::normalize (Geometry.cuh:35) */
static inline vec2 normalize(vec2 a) {
    double l = sqrt(a.x * a.x + a.y * a.y);
    if (!(fabs(l) < 1e-12)) { a.x /= l; a.y /= l; }
    return a;
}
/* toLeft, Geometry.cu:306-310 */
static inline int to_left(vec2 p, vec2 p0, vec2 p1) {
    vec2 a = normalize(sub(p1, p0)), b = normalize(sub(p, p0));
    return cross(a, b) > 0.0;
}
/* ICHDevice::Intersect, ICHDevice.cu:975-980 */
static inline double intersect(vec2 v0, vec2 v1, vec2 p0, vec2 p1) {
    double a00 = p0.x - p1.x, a01 = v1.x - v0.x, b0 = v1.x - p1.x;
    double a10 = p0.y - p1.y, a11 = v1.y - v0.y, b1 = v1.y - p1.y;
    return (b0 * a11 - b1 * a01) / (a00 * a11 - a10 * a01);
}

/* ------------------------------------------------------------ ICH types */
typedef struct {  /* ICHDevice::Window, ICHDevice.cuh:16-50 */
    int edge;
    double b0, b1, d0, d1, psd, minDist;
    int psrc;
    int birth;
    int level;
} Win;
typedef struct {  /* ICHDevice::PseudoWindow, ICHDevice.cuh:52-63 */
    int vert;
    double dist;
    unsigned birth;
    unsigned level;
} PWin;
typedef struct { double dist, x; int psrc; } Split;  /* ICHDevice.cuh:65-72 */
typedef struct { signed char birth; double dist; int isSource; int enterEdge; } VInfo; /* :74-86 */

static inline void calc_min_dist(Win* w) {  /* ICHDevice.cuh:30-39 */
    double wLen = w->b1 - w->b0;
    double xProj = (w->d0 * w->d0 + wLen * wLen - w->d1 * w->d1) / (2 * wLen);
    if (xProj < 0.0) w->minDist = w->d0 + w->psd;
    else if (xProj > wLen) w->minDist = w->d1 + w->psd;
    else w->minDist = sqrt(fabs(w->d0 * w->d0 - xProj * xProj)) + w->psd;
}
static inline vec2 flat_src(const Win* w) {  /* ICHDevice.cuh:41-49 */
    double wLen = w->b1 - w->b0;
    vec2 s;
    s.x = (w->d0 * w->d0 + wLen * wLen - w->d1 * w->d1) / (2.0 * wLen);
    s.y = sqrt(fabs(w->d0 * w->d0 - s.x * s.x));
    s.x += w->b0;
    return s;
}

/* 1-based binary min-heap over a caller buffer; push is dropped when full
 * (PriorityQueue.cuh:48-105).  Instantiated for both item types. */
#define DEFINE_HEAP(NAME, T)                                                           \
    typedef struct { double key; T item; } NAME##_it;                                  \
    typedef struct { NAME##_it* d; int tail; int maxSize; } NAME;                      \
    static inline void NAME##_push(NAME* q, T item, double key) {                      \
        if (q->tail - 1 >= q->maxSize) return;                                         \
        ++q->tail;                                                                     \
        int cur = q->tail - 1, p = cur / 2;                                            \
        while (p > 0 && q->d[p].key > key) { q->d[cur] = q->d[p]; cur = p; p = cur / 2; } \
        q->d[cur].item = item; q->d[cur].key = key;                                    \
    }                                                                                  \
    static inline T NAME##_pop(NAME* q) {                                              \
        T ret = q->d[1].item;                                                          \
        --q->tail;                                                                     \
        NAME##_it top = q->d[q->tail];                                                 \
        int cur = 1, l = 2, r = 3, mc = -1;                                            \
        if (r < q->tail) mc = q->d[l].key < q->d[r].key ? l : r;                       \
        else if (l < q->tail) mc = l;                                                  \
        while (mc != -1 && q->d[mc].key < top.key) {                                   \
            q->d[cur] = q->d[mc]; cur = mc; l = cur * 2; r = cur * 2 + 1;              \
            if (r < q->tail) mc = q->d[l].key < q->d[r].key ? l : r;                   \
            else if (l < q->tail) mc = l;                                              \
            else mc = -1;                                                              \
        }                                                                              \
        q->d[cur] = top;                                                               \
        return ret;                                                                    \
    }
DEFINE_HEAP(WinQ, Win)
DEFINE_HEAP(PsQ, PWin)

/* Fixed-size open-addressing table, golden-ratio hash, linear probing, no
 * deletion; slot `size` is the shared overflow sink (MyHashTable.cuh:8-117).
 * operator[] records the key in the slot it returns, even for reads. */
typedef struct { VInfo item; int index; } VSlot;
typedef struct { Split item; int index; } SSlot;

static inline unsigned gold_hash(unsigned index, unsigned size) {  /* MyHashTable.cuh:114-117 */
    return (unsigned)(int)(((double)index * 0.618033989 - (double)(int)((double)index * 0.618033989)) *
                           (double)size);
}
#define DEFINE_TABLE(NAME, SLOT)                                                       \
    static inline unsigned NAME##_key(SLOT* d, unsigned size, unsigned index) {        \
        unsigned key = gold_hash(index, size);                                         \
        unsigned i = 0;                                                                \
        for (; i < size; ++i) {                                                        \
            if (d[key].index == (int)index || d[key].index == -1) break;               \
            key = (key + 1) % size;                                                    \
        }                                                                              \
        if (i == size) key = size;                                                     \
        return key;                                                                    \
    }

DEFINE_TABLE(vt, VSlot)
DEFINE_TABLE(st, SSlot)

typedef struct {
    const om_mesh* m;
    VSlot* vd; unsigned vsize;
    SSlot* sd; unsigned ssize;
    WinQ wq; PsQ pq;
    int source;
    int total;          /* totalCalcVertNum */
    int numOfWinGen, maxWinQ, maxPsQ;
    int flags;
    int pathPassVert;
} Ich;

static inline VInfo* vget(Ich* s, unsigned v) { return &s->vd[vt_key(s->vd, s->vsize, v)].item; }
static inline VInfo* vput(Ich* s, unsigned v) {
    unsigned k = vt_key(s->vd, s->vsize, v);
    if (k == s->vsize) s->flags |= 1;
    s->vd[k].index = (int)v;
    return &s->vd[k].item;
}
static inline Split* sget(Ich* s, unsigned e) { return &s->sd[st_key(s->sd, s->ssize, e)].item; }
static inline Split* sput(Ich* s, unsigned e) {
    unsigned k = st_key(s->sd, s->ssize, e);
    if (k == s->ssize) s->flags |= 1;
    s->sd[k].index = (int)e;
    return &s->sd[k].item;
}

/* ICHDevice::Clear, ICHDevice.cu:487-523 */
static void ich_clear(Ich* s) {
    s->wq.tail = 1; s->pq.tail = 1;
    for (unsigned i = 0; i < s->ssize + 1; ++i) {
        s->sd[i].item.dist = DBL_MAX; s->sd[i].item.x = DBL_MAX; s->sd[i].item.psrc = -1;
        s->sd[i].index = -1;
    }
    for (unsigned i = 0; i < s->vsize + 1; ++i) {
        s->vd[i].item.birth = -1; s->vd[i].item.dist = DBL_MAX; s->vd[i].item.enterEdge = -1;
        s->vd[i].item.isSource = 0; s->vd[i].index = -1;
    }
    s->numOfWinGen = 0; s->maxWinQ = 0; s->maxPsQ = 0; s->total = 0; s->flags = 0;
}

/* ICHDevice::Initialize for a vertex source, ICHDevice.cu:525-581 */
static void ich_initialize(Ich* s) {
    const om_mesh* m = s->m;
    int src = s->source;
    int start = m->first[src], cur = start;
    if (start < 0) { s->flags |= 2; return; }
    do {
        int op = m->next[cur];
        Win w;
        w.edge = op; w.b0 = 0.0; w.b1 = m->len[op];
        w.d0 = m->len[cur]; w.d1 = m->len[m->prev[cur]];
        w.psd = 0.0; calc_min_dist(&w);
        w.psrc = src; w.birth = 0; w.level = 0;
        WinQ_push(&s->wq, w, w.minDist);
        ++s->numOfWinGen;
        int opv = m->v1[cur];
        if (m->len[cur] > vput(s, opv)->dist) {
            cur = m->twin[cur];
            if (cur != -1) cur = m->next[cur];
            continue;
        }
        VInfo* vi = vput(s, opv);
        vi->birth = 0; vi->dist = m->len[cur]; vi->enterEdge = m->twin[cur];
        if (m->angle[opv] < 2.0 * REF_PI) {
            cur = m->twin[cur];
            if (cur != -1) cur = m->next[cur];
            continue;
        }
        PWin pw;
        pw.vert = opv; pw.dist = m->len[cur];
        pw.birth = (unsigned)(int)vget(s, opv)->birth; pw.level = 0;
        PsQ_push(&s->pq, pw, pw.dist);
        cur = m->twin[cur];
        if (cur != -1) cur = m->next[cur];
    } while (cur != start && cur != -1);
    VInfo* sv = vput(s, src);
    sv->birth = 0; sv->dist = 0.0; sv->enterEdge = -1; sv->isSource = 1;
}

/* ICHDevice::IsValidWindow, ICHDevice.cu:906-955 */
static int is_valid(Ich* s, const Win* w, int isLeft) {
    const om_mesh* m = s->m;
    if (w->b1 <= w->b0) return 0;
    int e = w->edge;
    int v1 = m->v0[e], v2 = m->v1[e], v3 = m->v1[m->next[e]];
    double l0 = m->len[e], l1 = m->len[m->next[e]], l2 = m->len[m->next[m->next[e]]];
    vec2 p3;
    p3.x = (l2 * l2 + l0 * l0 - l1 * l1) / (2.0 * l0);
    p3.y = sqrt(fabs(l2 * l2 - p3.x * p3.x));
    vec2 A = mk(w->b0, 0.0), B = mk(w->b1, 0.0);
    vec2 src = flat_src(w);
    double dv1 = vget(s, v1)->dist, dv2 = vget(s, v2)->dist, dv3 = vget(s, v3)->dist;
    if (w->psd + len2d(sub(src, B)) > dv1 + w->b1 &&
        (w->psd + len2d(sub(src, B))) / (dv1 + w->b1) - 1.0 > 0.0)
        return 0;
    if (w->psd + len2d(sub(src, A)) > dv2 + l0 - w->b0 &&
        (w->psd + len2d(sub(src, A))) / (dv2 + l0 - w->b0) - 1.0 > 0.0)
        return 0;
    if (isLeft) {
        if (w->psd + len2d(sub(src, A)) > dv3 + len2d(sub(p3, A)) &&
            (w->psd + len2d(sub(src, A))) / (dv3 + len2d(sub(p3, A))) - 1.0 > 0.0)
            return 0;
    } else {
        if (w->psd + len2d(sub(src, B)) > dv3 + len2d(sub(p3, B)) &&
            (w->psd + len2d(sub(src, B))) / (dv3 + len2d(sub(p3, B))) - 1.0 > RELATIVE_ERROR)
            return 0;
    }
    return 1;
}

/* ICHDevice::BuildWindow, ICHDevice.cu:957-973 */
static void build_window(const om_mesh* m, const Win* f, int edge, double t0, double t1, vec2 v0,
                         vec2 v1, Win* w) {
    vec2 src = flat_src(f);
    w->edge = edge;
    w->b0 = (1 - t0) * m->len[edge];
    w->b1 = (1 - t1) * m->len[edge];
    w->d0 = len2d(sub(src, add(scl(t0, v0), scl(1 - t0, v1))));
    w->d1 = len2d(sub(src, add(scl(t1, v0), scl(1 - t1, v1))));
    w->psd = f->psd;
    calc_min_dist(w);
    w->psrc = f->psrc;
    w->birth = f->birth;
    w->level = f->level + 1;
}

/* ICHDevice::PropagateWindow, ICHDevice.cu:618-726 */
static void propagate(Ich* s, const Win* win) {
    const om_mesh* m = s->m;
    int e0 = m->twin[win->edge];
    if (e0 == -1) return;
    int e1 = m->next[e0], e2 = m->next[e1];
    int opv = m->v1[e1];
    vec2 src = flat_src(win);
    vec2 left = mk(win->b0, 0.0), right = mk(win->b1, 0.0);
    double l0 = m->len[e0], l1 = m->len[e1], l2 = m->len[e2];
    vec2 v0 = mk(0.0, 0.0), v1 = mk(l0, 0.0), v2;
    v2.x = (l1 * l1 + l0 * l0 - l2 * l2) / (2.0 * l0);
    v2.y = -sqrt(fabs(l1 * l1 - v2.x * v2.x));
    double interX = v2.x - v2.y * (v2.x - src.x) / (v2.y - src.y);
    Win L, R;
    int hasL = 1, hasR = 1;
    if (interX <= left.x) {
        hasL = 0;
        double t0 = intersect(src, left, v2, v1);
        double t1 = intersect(src, right, v2, v1);
        build_window(m, win, e2, t0, t1, v2, v1, &R);
        if (!is_valid(s, &R, 0)) hasR = 0;
    } else if (interX >= right.x) {
        hasR = 0;
        double t0 = intersect(src, left, v0, v2);
        double t1 = intersect(src, right, v0, v2);
        build_window(m, win, e1, t0, t1, v0, v2, &L);
        if (!is_valid(s, &L, 1)) hasL = 0;
    } else {
        double direct = len2d(sub(v2, src));
        double sd = sget(s, e0)->dist;
        if (direct + win->psd > sd && (direct + win->psd) / sget(s, e0)->dist - 1.0 > RELATIVE_ERROR) {
            hasL = sget(s, e0)->x < interX;
            hasR = !hasL;
        } else {
            if (direct + win->psd < sget(s, e0)->dist) {
                Split* sp = sput(s, e0);
                sp->dist = direct + win->psd;
                sp->psrc = win->psrc;
                sp->x = l0 - interX;
            }
            if (direct + win->psd < vget(s, opv)->dist) {
                if (vget(s, opv)->dist == DBL_MAX) ++s->total;
                VInfo* vi = vput(s, opv);
                vi->birth = (signed char)(vi->birth + 1);
                vi->dist = direct + win->psd;
                vi->enterEdge = e0;
                if (m->angle[opv] > 2.0 * REF_PI) {
                    PWin pw;
                    pw.vert = opv; pw.dist = vget(s, opv)->dist;
                    pw.birth = (unsigned)(int)vget(s, opv)->birth;
                    pw.level = (unsigned)(win->level + 1);
                    PsQ_push(&s->pq, pw, pw.dist);
                }
            }
        }
        if (hasL) {
            double t0 = intersect(src, left, v0, v2);
            build_window(m, win, e1, t0, 0.0, v0, v2, &L);
            if (!is_valid(s, &L, 1)) hasL = 0;
        }
        if (hasR) {
            double t1 = intersect(src, right, v2, v1);
            build_window(m, win, e2, 1.0, t1, v2, v1, &R);
            if (!is_valid(s, &R, 0)) hasR = 0;
        }
    }
    if (hasL) { ++s->numOfWinGen; WinQ_push(&s->wq, L, L.minDist); }
    if (hasR) { ++s->numOfWinGen; WinQ_push(&s->wq, R, R.minDist); }
}

/* Corner angle walk shared by GenSubWinsForPseudoSrcFrom* (ICHDevice.cu:824-857, 870-903). */
static inline double corner(const om_mesh* m, int a, int b, int c) {
    double L0 = m->len[a], L1 = m->len[b], L2 = m->len[c];
    double ca = (L0 * L0 + L1 * L1 - L2 * L2) / (2.0 * L0 * L1);
    if (ca > 1.0) ca = 1.0; else if (ca < -1.0) ca = -1.0;
    return acos(ca);
}
static void fan_walk(Ich* s, int leftStart, int rightStart, double angle0, double angle1, int* startEdge,
                     int* endEdge) {
    const om_mesh* m = s->m;
    *startEdge = -1; *endEdge = -1;
    int cur = leftStart;
    long long guard = 0;
    while (angle0 < REF_PI && cur != -1) {
        int op = m->next[cur], nx = m->next[op];
        angle0 += corner(m, cur, nx, op);
        cur = m->twin[nx];
        if (++guard > FAN_GUARD) { s->flags |= 2; return; }
    }
    if (cur != -1) *startEdge = m->next[m->twin[cur]];
    cur = rightStart;
    while (angle1 < REF_PI && cur != -1) {
        int nx = m->next[cur], op = m->next[nx];
        angle1 += corner(m, cur, nx, op);
        cur = m->twin[nx];
        if (++guard > FAN_GUARD) { s->flags |= 2; return; }
    }
    if (cur != -1) *endEdge = m->twin[m->next[m->next[m->twin[cur]]]];
}

/* ICHDevice::GenSubWinsForPseudoSrcFromWindow, ICHDevice.cu:795-858 */
static void from_window(Ich* s, const PWin* pw, int* startEdge, int* endEdge) {
    const om_mesh* m = s->m;
    int e0 = vget(s, pw->vert)->enterEdge, e1 = m->next[e0], e2 = m->next[e1];
    double l0 = m->len[e0], l1 = m->len[e1], l2 = m->len[e2];
    vec2 enter = mk(l0 - sget(s, e0)->x, 0.0);
    vec2 v0 = mk(0.0, 0.0), v1 = mk(l0, 0.0), v2;
    v2.x = (l1 * l1 + l0 * l0 - l2 * l2) / (2.0 * l0);
    v2.y = -sqrt(fabs(l1 * l1 - v2.x * v2.x));
    double a0 = dot(sub(enter, v2), sub(v0, v2)) / len2d(sub(enter, v2)) / l1;
    double a1 = dot(sub(enter, v2), sub(v1, v2)) / len2d(sub(enter, v2)) / l2;
    if (a0 > 1.0) a0 = 1.0; else if (a0 < -1.0) a0 = -1.0;
    if (a1 > 1.0) a1 = 1.0; else if (a1 < -1.0) a1 = -1.0;
    a0 = acos(a0); a1 = acos(a1);
    fan_walk(s, m->twin[e1], m->twin[e2], a0, a1, startEdge, endEdge);
}

/* ICHDevice::GenSubWinsForPseudoSrcFromPseudoSrc, ICHDevice.cu:860-904 */
static void from_pseudo(Ich* s, const PWin* pw, int* startEdge, int* endEdge) {
    int ee = vget(s, pw->vert)->enterEdge;
    fan_walk(s, ee, s->m->twin[ee], 0.0, 0.0, startEdge, endEdge);
}

/* ICHDevice::GenSubWinsForPseudoSrc, ICHDevice.cu:728-793 */
static void gen_sub_wins(Ich* s, const PWin* pw) {
    const om_mesh* m = s->m;
    int startEdge, endEdge;
    VInfo vi = *vget(s, pw->vert);
    if (vi.enterEdge == -1 && vi.birth != -1) {
        startEdge = m->first[pw->vert];
        endEdge = startEdge;
    } else if (vi.enterEdge >= 0 && m->v0[vi.enterEdge] == (int)pw->vert) {
        from_pseudo(s, pw, &startEdge, &endEdge);
    } else if (vi.enterEdge >= 0 && m->v1[m->next[vi.enterEdge]] == (int)pw->vert) {
        from_window(s, pw, &startEdge, &endEdge);
    } else {
        s->flags |= 2;  /* assert(false) in the reference */
        return;
    }
    if (s->flags & 2) return;
    long long guard = 0;
    do {
        if (startEdge < 0) { s->flags |= 2; break; }  /* reference indexes edges[-1] here */
        Win w;
        w.edge = m->next[startEdge];
        w.b0 = 0.0; w.b1 = m->len[w.edge];
        w.d0 = m->len[startEdge]; w.d1 = m->len[m->next[w.edge]];
        w.psd = pw->dist; calc_min_dist(&w);
        w.psrc = (int)pw->vert; w.birth = (int)pw->birth; w.level = (int)pw->level + 1;
        WinQ_push(&s->wq, w, w.minDist);
        ++s->numOfWinGen;
        startEdge = m->twin[m->next[m->next[startEdge]]];
        if (++guard > FAN_GUARD) { s->flags |= 2; break; }
    } while (startEdge != endEdge);

    int start = m->first[pw->vert], cur = start;
    do {
        int opv = m->v1[cur];
        if (m->angle[opv] < 2.0 * REF_PI || vget(s, opv)->dist < pw->dist + m->len[cur]) {
            cur = m->twin[cur];
            if (cur != -1) cur = m->next[cur];
            continue;
        }
        if (vget(s, opv)->dist == DBL_MAX) ++s->total;
        VInfo* o = vput(s, opv);
        o->dist = pw->dist + m->len[cur];
        o->birth = (signed char)(o->birth + 1);
        o->enterEdge = m->twin[cur];
        PWin c;
        c.vert = (unsigned)opv; c.dist = vget(s, opv)->dist;
        c.birth = (unsigned)(int)vget(s, opv)->birth; c.level = pw->level;
        PsQ_push(&s->pq, c, c.dist);
        cur = m->twin[cur];
        if (cur != -1) cur = m->next[cur];
    } while (cur != start && cur != -1);
}

/* ICHDevice::Execute, ICHDevice.cu:67-119 (vertex source: no stored windows). */
static void ich_execute(Ich* s, int K) {
    const om_mesh* m = s->m;
    ich_initialize(s);
    long long guard = 0;
    while (s->wq.tail != 1 || s->pq.tail != 1) {
        if (++guard > WATCHDOG || (s->flags & 2)) { s->flags |= 2; break; }
        if (s->wq.tail - 1 > s->maxWinQ) s->maxWinQ = s->wq.tail - 1;
        if (s->pq.tail - 1 > s->maxPsQ) s->maxPsQ = s->pq.tail - 1;
        /* Stale tops: a window or pseudo-source whose birth time no longer
         * matches its pseudo-source vertex is outdated.  (The pseudo loop's
         * guard at :84 reads winQ.top().pseudoSrcId, always a vertex id here.) */
        while (s->wq.tail != 1 && s->wq.d[1].item.psrc < m->nv &&
               s->wq.d[1].item.birth != (int)vget(s, s->wq.d[1].item.psrc)->birth)
            WinQ_pop(&s->wq);
        while (s->pq.tail != 1 && s->pq.d[1].item.birth != (unsigned)(int)vget(s, s->pq.d[1].item.vert)->birth)
            PsQ_pop(&s->pq);
        if (s->wq.tail != 1 && (s->pq.tail == 1 || s->wq.d[1].item.minDist < s->pq.d[1].item.dist)) {
            Win w = WinQ_pop(&s->wq);
            if (w.level > m->nf) continue;
            propagate(s, &w);
        } else if (s->pq.tail != 1 && (s->wq.tail == 1 || s->wq.d[1].item.minDist >= s->pq.d[1].item.dist)) {
            PWin p = PsQ_pop(&s->pq);
            if (p.level >= (unsigned)m->nf) continue;
            gen_sub_wins(s, &p);
        }
        if (K != -1 && s->total >= K) break;
    }
}

/* ICHDevice::BuildGeodesicPathTo(vertex), ICHDevice.cu:336-480 */
static void trace(Ich* s, int vert, unsigned* nextToSrcEdge, double* nextToSrcX, unsigned* nextToDstEdge,
                  double* nextToDstX) {
    const om_mesh* m = s->m;
    s->pathPassVert = 0;
    *nextToSrcEdge = (unsigned)-1; *nextToDstEdge = (unsigned)-1;
    int curVert = vert;
    long long guard = 0, tcap = 4LL * m->nf + 64;
    while (vget(s, curVert)->dist != 0.0) {
        if (++guard > tcap) { s->flags |= 2; s->pathPassVert = 1; return; }
        int enterEdge = vget(s, curVert)->enterEdge;
        if (enterEdge == -1) {
            if (*nextToDstEdge == (unsigned)-1) { *nextToDstEdge = m->first[curVert]; *nextToDstX = 0.0; }
            else { *nextToSrcEdge = m->first[curVert]; *nextToSrcX = 0.0; }
            s->pathPassVert = 1;
            return;
        } else if (m->v0[enterEdge] == curVert) {
            int nextVert = m->v1[enterEdge];
            if (!vget(s, nextVert)->isSource) {
                if (*nextToDstEdge == (unsigned)-1) { *nextToDstEdge = m->next[enterEdge]; *nextToDstX = 0.0; }
                else { *nextToSrcEdge = m->next[enterEdge]; *nextToSrcX = 0.0; }
                s->pathPassVert = 1;
            }
            curVert = nextVert;
        } else {
            int gid = enterEdge;
            double gpos = sget(s, enterEdge)->x;
            if (*nextToDstEdge == (unsigned)-1) { *nextToDstEdge = gid; *nextToDstX = gpos; }
            else { *nextToSrcEdge = gid; *nextToSrcX = gpos; }
            int opv = m->twin[gid];
            if (opv == -1) { s->flags |= 2; return; }
            opv = m->v1[m->next[opv]];
            double l0 = m->len[gid], l1 = m->len[m->next[gid]], l2 = m->len[m->next[m->next[gid]]];
            vec2 last, curp;
            last.x = (l1 * l1 + l0 * l0 - l2 * l2) / (2.0 * l0);
            last.y = -sqrt(fabs(l1 * l1 - last.x * last.x));
            curp = mk(l0 - gpos, 0.0);
            /* :414-417 with pseudoSrcId < vertNum (vertex sources only) */
            unsigned psrc = (unsigned)sget(s, enterEdge)->psrc;
            if (psrc >= (unsigned)m->nv) { s->flags |= 2; return; }
            while (opv != (int)psrc) {
                if (++guard > tcap) { s->flags |= 2; s->pathPassVert = 1; return; }
                int e0 = m->twin[gid], e1 = m->next[e0], e2 = m->next[e1];
                double L0 = m->len[e0], L1 = m->len[e1], L2 = m->len[e2];
                vec2 ov;
                ov.x = (L0 * L0 + L2 * L2 - L1 * L1) / (2.0 * L0);
                ov.y = sqrt(fabs(L2 * L2 - ov.x * ov.x));
                if (to_left(ov, last, curp)) {
                    vec2 p0, p1;
                    p0.x = (L2 * L2 + L1 * L1 - L0 * L0) / (2.0 * L1);
                    p0.y = -sqrt(fabs(L2 * L2 - p0.x * p0.x));
                    p1 = mk(L1, 0.0);
                    vec2 nl = add(scl(gpos / L0, p0), scl(1.0 - gpos / L0, p1));
                    gpos = intersect(last, curp, mk(L0, 0.0), ov);
                    gpos = (1.0 - gpos) * L1;
                    gid = e1;
                    curp = mk(L1 - gpos, 0.0);
                    last = nl;
                } else {
                    vec2 p0 = mk(0.0, 0.0), p1;
                    p1.x = (L2 * L2 + L0 * L0 - L1 * L1) / (2.0 * L2);
                    p1.y = -sqrt(fabs(L0 * L0 - p1.x * p1.x));
                    vec2 nl = add(scl(gpos / L0, p0), scl(1.0 - gpos / L0, p1));
                    gpos = intersect(last, curp, ov, mk(0.0, 0.0));
                    gpos = (1.0 - gpos) * L2;
                    gid = e2;
                    curp = mk(L2 - gpos, 0.0);
                    last = nl;
                }
                *nextToSrcEdge = gid; *nextToSrcX = gpos;
                opv = m->twin[gid];
                if (opv == -1) { s->flags |= 2; return; }  /* reference reads edges[-1] */
                opv = m->v1[m->next[opv]];
            }
            if (!vget(s, opv)->isSource) {
                *nextToSrcEdge = m->first[opv]; *nextToSrcX = 0.0;
                s->pathPassVert = 1;
            }
            curVert = opv;
        }
    }
}

/* ------------------------------------------------------------- drivers */
typedef struct {
    const om_mesh* m;
    int K;
    unsigned vsize, ssize;
    int wcap, pcap;
    const int32_t* sources;
    int nsrc;
    int32_t* tails;
    om_node* nodes;
    int32_t* stats;
    double* dist;       /* om_ich_distances mode */
    int emit;
    int next;
    pthread_mutex_t* lock;
} Job;

static void* worker(void* arg) {
    Job* j = (Job*)arg;
    const om_mesh* m = j->m;
    Ich s;
    memset(&s, 0, sizeof(s));
    s.m = m;
    s.vsize = j->vsize; s.ssize = j->ssize;
    s.vd = (VSlot*)malloc(sizeof(VSlot) * (j->vsize + 1));
    s.sd = (SSlot*)malloc(sizeof(SSlot) * (j->ssize + 1));
    s.wq.d = (WinQ_it*)malloc(sizeof(WinQ_it) * (size_t)(j->wcap + 2));
    s.pq.d = (PsQ_it*)malloc(sizeof(PsQ_it) * (size_t)(j->pcap + 2));
    s.wq.maxSize = j->wcap; s.pq.maxSize = j->pcap;
    for (;;) {
        pthread_mutex_lock(j->lock);
        int r = j->next++;
        pthread_mutex_unlock(j->lock);
        if (r >= j->nsrc) break;
        int src = j->sources[r];
        ich_clear(&s);
        s.source = src;
        ich_execute(&s, j->K);
        if (j->emit) {
            /* SVG.cu:42-75 */
            int tail = 0;
            om_node* row = j->nodes + (size_t)j->K * r;
            for (int v = 0; v < m->nv && j->K > 0; ++v) {
                if (vget(&s, v)->dist == DBL_MAX) continue;
                if (v == src) continue;
                unsigned se, de;
                double sx = 0.0, dx = 0.0;
                trace(&s, v, &se, &sx, &de, &dx);
                if (s.pathPassVert) continue;
                if (se == (unsigned)-1) { se = de; sx = dx; }
                row[tail].adj = v; row[tail].pad_ = 0;
                row[tail].dist = vget(&s, v)->dist;
                row[tail].next_to_src_edge = se; row[tail].next_to_src_x = sx;
                row[tail].next_to_dst_edge = de; row[tail].next_to_dst_x = dx;
                ++tail;
                if (tail == j->K) break;
            }
            j->tails[r] = tail;
        } else {
            double* d = j->dist + (size_t)m->nv * r;
            for (int v = 0; v < m->nv; ++v) d[v] = vget(&s, v)->dist;
        }
        if (j->stats) {
            int32_t* st = j->stats + 5 * (size_t)r;
            st[0] = s.numOfWinGen; st[1] = s.maxWinQ; st[2] = s.maxPsQ; st[3] = s.total; st[4] = s.flags;
        }
    }
    free(s.vd); free(s.sd); free(s.wq.d); free(s.pq.d);
    return NULL;
}

static double now_s(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

static double run_jobs(Job* j, int nthreads) {
    pthread_mutex_t lock = PTHREAD_MUTEX_INITIALIZER;
    j->lock = &lock;
    j->next = 0;
    if (nthreads <= 0) nthreads = (int)sysconf(_SC_NPROCESSORS_ONLN);
    if (nthreads < 1) nthreads = 1;
    if (nthreads > j->nsrc) nthreads = j->nsrc > 0 ? j->nsrc : 1;
    double t0 = now_s();
    pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)nthreads);
    for (int t = 1; t < nthreads; ++t) pthread_create(&th[t], NULL, worker, j);
    worker(j);
    for (int t = 1; t < nthreads; ++t) pthread_join(th[t], NULL);
    free(th);
    return now_s() - t0;
}

double om_build(const om_mesh* m, int K, unsigned split_coef, unsigned vert_coef, int win_cap,
                int pseudo_cap, const int32_t* sources, int nsrc, int nthreads, int32_t* tails,
                om_node* nodes, int32_t* stats) {
    Job j;
    memset(&j, 0, sizeof(j));
    j.m = m; j.K = K; j.vsize = (unsigned)K * vert_coef; j.ssize = (unsigned)K * split_coef;
    j.wcap = win_cap; j.pcap = pseudo_cap; j.sources = sources; j.nsrc = nsrc;
    j.tails = tails; j.nodes = nodes; j.stats = stats; j.emit = 1;
    return run_jobs(&j, nthreads);
}

double om_ich_distances(const om_mesh* m, int K, unsigned split_size, unsigned vert_size,
                        int win_cap, int pseudo_cap, const int32_t* sources, int nsrc,
                        int nthreads, double* dist, int32_t* stats) {
    Job j;
    memset(&j, 0, sizeof(j));
    j.m = m; j.K = K; j.vsize = vert_size; j.ssize = split_size;
    j.wcap = win_cap; j.pcap = pseudo_cap; j.sources = sources; j.nsrc = nsrc;
    j.dist = dist; j.stats = stats; j.emit = 0;
    return run_jobs(&j, nthreads);
}

/* --------------------------------------------------------- graph search */
/* Addressable binary heap (PriorityQueueWithHandle.cuh:48-135): each item
 * keeps a pointer to its owner's handle so decrease-key can find it. */
typedef struct { double key; int item; int* back; } HItem;
typedef struct { HItem* d; int tail; } HHeap;

static void hh_push(HHeap* q, int item, int* back, double key) {
    ++q->tail;
    int cur = q->tail - 1, p = cur / 2;
    while (p > 0 && q->d[p].key > key) {
        q->d[cur] = q->d[p]; *(q->d[cur].back) = cur; cur = p; p = cur / 2;
    }
    q->d[cur].item = item; q->d[cur].key = key; q->d[cur].back = back; *back = cur;
}
static int hh_pop(HHeap* q) {
    int ret = q->d[1].item;
    *(q->d[1].back) = -1;
    --q->tail;
    HItem top = q->d[q->tail];
    int cur = 1, l = 2, r = 3, mc = -1;
    if (r < q->tail) mc = q->d[l].key < q->d[r].key ? l : r;
    else if (l < q->tail) mc = l;
    while (mc != -1 && q->d[mc].key < top.key) {
        q->d[cur] = q->d[mc]; *(q->d[cur].back) = cur;
        cur = mc; l = cur * 2; r = cur * 2 + 1;
        if (r < q->tail) mc = q->d[l].key < q->d[r].key ? l : r;
        else if (l < q->tail) mc = l;
        else mc = -1;
    }
    /* Written back unconditionally, as the reference does: popping the last
     * item leaves that item's handle at 1, not -1 (harmless under a
     * consistent heuristic: a popped node is never relaxed again). */
    q->d[cur] = top;
    *(q->d[cur].back) = cur;
    return ret;
}
static void hh_decrease(HHeap* q, int h, double key) {
    int cur = h, p = cur / 2;
    HItem it = q->d[cur];
    while (p > 0 && q->d[p].key > key) {
        q->d[cur] = q->d[p]; *(q->d[cur].back) = cur; cur = p; p = cur / 2;
    }
    q->d[cur] = it; q->d[cur].key = key; *(q->d[cur].back) = cur;
}

typedef struct { double dist; int parent; int src; int inpq; } GInfo;

/* SVG::Astar, SVG.cu:369-413 */
static void astar(const om_mesh* m, const int64_t* off, const int32_t* adj, const double* w, int t,
                  int isAstar, GInfo* g, HHeap* q) {
    while (q->tail != 1) {
        int cur = hh_pop(q);
        if (isAstar && cur == t) { q->tail = 1; break; }
        for (int64_t i = off[cur]; i < off[cur + 1]; ++i) {
            int a = adj[i];
            double nd = g[cur].dist + w[i];
            if (nd >= g[a].dist) continue;
            g[a].dist = nd; g[a].parent = cur; g[a].src = g[cur].src;
            double pri = isAstar ? nd + len3(&m->pos[3 * a], &m->pos[3 * t]) : nd;
            if (g[a].inpq == -1) hh_push(q, a, &g[a].inpq, pri);
            else hh_decrease(q, g[a].inpq, pri);
        }
    }
}

double om_sssd(const om_mesh* m, const int64_t* off, const int32_t* adj, const double* w, int n,
               const int32_t* s, const int32_t* t, double* dist_out) {
    int V = m->nv;
    GInfo* g = (GInfo*)malloc(sizeof(GInfo) * (size_t)V);
    HHeap q;
    q.d = (HItem*)malloc(sizeof(HItem) * (size_t)(V + 2));
    double t0 = now_s();
    for (int k = 0; k < n; ++k) {
        for (int i = 0; i < V; ++i) { g[i].dist = DBL_MAX; g[i].parent = -1; g[i].src = -1; g[i].inpq = -1; }
        q.tail = 1;
        int ss = s[k], tt = t[k];
        g[ss].dist = 0.0; g[ss].parent = -1; g[ss].src = ss;
        hh_push(&q, ss, &g[ss].inpq, 0.0 + len3(&m->pos[3 * ss], &m->pos[3 * tt]));
        astar(m, off, adj, w, tt, 1, g, &q);
        dist_out[k] = g[tt].dist;
    }
    double el = now_s() - t0;
    free(g); free(q.d);
    return el;
}

double om_msad(const om_mesh* m, const int64_t* off, const int32_t* adj, const double* w, int ns,
               const int32_t* srcs, const double* weights, double* dist_out, int32_t* src_out) {
    int V = m->nv;
    GInfo* g = (GInfo*)malloc(sizeof(GInfo) * (size_t)V);
    HHeap q;
    q.d = (HItem*)malloc(sizeof(HItem) * (size_t)(V + 2));
    for (int i = 0; i < V; ++i) { g[i].dist = DBL_MAX; g[i].parent = -1; g[i].src = -1; g[i].inpq = -1; }
    q.tail = 1;
    double t0 = now_s();
    /* SVG.cu:358-364: every listed source is pushed; a repeated source keeps
     * the weight of its last occurrence as its distance. */
    for (int i = 0; i < ns; ++i) {
        int v = srcs[i];
        g[v].dist = weights[i]; g[v].parent = -1; g[v].src = v;
        hh_push(&q, v, &g[v].inpq, weights[i]);
    }
    astar(m, off, adj, w, -1, 0, g, &q);
    double el = now_s() - t0;
    for (int v = 0; v < V; ++v) { dist_out[v] = g[v].dist; if (src_out) src_out[v] = g[v].src; }
    free(g); free(q.d);
    return el;
}
