/*
 * ORACLE — test infrastructure only (tests/, smoke() and the bench's CPU baseline).
 *
 * CPU closest-hit ray casting with the semantics the GPU backend promises for
 * rtcIntersect1's replacement (src/filianore/bvh/bvh.cpp:49-84):
 *   - watertight, double-sided triangle test (Woop, Benthin, Wald, "Watertight
 *     Ray/Triangle Intersection", JCGT 2013), evaluated in FP32 without contraction,
 *     with the paper's FP64 fallback when an edge function is exactly zero;
 *   - a hit needs tmin < t < tmax; equal t resolves to the lower triangle id, so the
 *     answer does not depend on traversal order;
 *   - triangle id = soup index (embree geomID, bvh.cpp:24-43 makes one geometry per
 *     triangle in insertion order); u, v = weights of v1 and v2.
 * The acceleration structure is a plain binary BVH built with a binned SAH; its
 * box test is made conservative (Ize, "Robust BVH Ray Traversal", JCGT 2013) so the
 * BVH answer equals brute force over all triangles (checked by the tests).
 *
 * Embree's own hit answer cannot be reproduced here: the embree submodule of the
 * reference (external/embree, .gitmodules:1-3) is empty and no embree is installed.
 */
#include "oracle.h"

#include <float.h>
#include <pthread.h>
#include <stdlib.h>

/* ---------------------------------------------------------------- watertight test */

void orc_ray_precompute(const float *o_tmin, const float *d_tmax, orc_ray *r) {
    r->o[0] = o_tmin[0]; r->o[1] = o_tmin[1]; r->o[2] = o_tmin[2]; r->tmin = o_tmin[3];
    r->d[0] = d_tmax[0]; r->d[1] = d_tmax[1]; r->d[2] = d_tmax[2]; r->tmax = d_tmax[3];
    float ax = fabsf(r->d[0]), ay = fabsf(r->d[1]), az = fabsf(r->d[2]);
    int kz = (ax > ay) ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
    int kx = kz + 1; if (kx == 3) kx = 0;
    int ky = kx + 1; if (ky == 3) ky = 0;
    if (r->d[kz] < 0.f) { int tmp = kx; kx = ky; ky = tmp; }
    r->kx = kx; r->ky = ky; r->kz = kz;
    r->Sx = r->d[kx] / r->d[kz];
    r->Sy = r->d[ky] / r->d[kz];
    r->Sz = 1.f / r->d[kz];
    r->valid = (r->d[kz] != 0.f) && !isnan(r->d[kz]);
    for (int i = 0; i < 3; ++i) r->inv_d[i] = 1.f / r->d[i];
}

int orc_intersect_watertight(const orc_ray *r, const float *v, float *t_out, float *u_out, float *v_out) {
    const int kx = r->kx, ky = r->ky, kz = r->kz;
    float A[3], B[3], C[3];
    for (int i = 0; i < 3; ++i) {
        A[i] = v[i] - r->o[i];
        B[i] = v[3 + i] - r->o[i];
        C[i] = v[6 + i] - r->o[i];
    }
    const float Ax = A[kx] - r->Sx * A[kz];
    const float Ay = A[ky] - r->Sy * A[kz];
    const float Bx = B[kx] - r->Sx * B[kz];
    const float By = B[ky] - r->Sy * B[kz];
    const float Cx = C[kx] - r->Sx * C[kz];
    const float Cy = C[ky] - r->Sy * C[kz];
    float U = Cx * By - Cy * Bx;
    float V = Ax * Cy - Ay * Cx;
    float W = Bx * Ay - By * Ax;
    if (U == 0.f || V == 0.f || W == 0.f) {
        U = (float)((double)Cx * (double)By - (double)Cy * (double)Bx);
        V = (float)((double)Ax * (double)Cy - (double)Ay * (double)Cx);
        W = (float)((double)Bx * (double)Ay - (double)By * (double)Ax);
    }
    if ((U < 0.f || V < 0.f || W < 0.f) && (U > 0.f || V > 0.f || W > 0.f)) return 0;
    const float det = U + V + W;
    if (det == 0.f) return 0;
    const float Az = r->Sz * A[kz];
    const float Bz = r->Sz * B[kz];
    const float Cz = r->Sz * C[kz];
    const float T = U * Az + V * Bz + W * Cz;
    const float t = T / det;
    if (!(t > r->tmin)) return 0;
    *t_out = t;
    *u_out = V / det;
    *v_out = W / det;
    return 1;
}

/* ---------------------------------------------------------------- BVH build */

typedef struct {
    float bmin[3], bmax[3];
    int32_t left;   /* internal: index of left child (right = left + 1); leaf: first prim */
    int32_t count;  /* 0 = internal, >0 = leaf size */
} orc_node;

struct orc_bvh {
    const float *tris; /* borrowed soup, n*9 */
    uint32_t n;
    orc_node *nodes;
    uint32_t n_nodes;
    uint32_t *prims;
};

typedef struct { float bmin[3], bmax[3]; } box3;

static void box_empty(box3 *b) {
    for (int i = 0; i < 3; ++i) { b->bmin[i] = FLT_MAX; b->bmax[i] = -FLT_MAX; }
}
static void box_grow_pt(box3 *b, const float *p) {
    for (int i = 0; i < 3; ++i) {
        if (p[i] < b->bmin[i]) b->bmin[i] = p[i];
        if (p[i] > b->bmax[i]) b->bmax[i] = p[i];
    }
}
static void box_grow(box3 *b, const box3 *o) {
    for (int i = 0; i < 3; ++i) {
        if (o->bmin[i] < b->bmin[i]) b->bmin[i] = o->bmin[i];
        if (o->bmax[i] > b->bmax[i]) b->bmax[i] = o->bmax[i];
    }
}
static float box_area(const box3 *b) {
    float dx = b->bmax[0] - b->bmin[0], dy = b->bmax[1] - b->bmin[1], dz = b->bmax[2] - b->bmin[2];
    if (dx < 0 || dy < 0 || dz < 0) return 0.f;
    return 2.f * (dx * dy + dy * dz + dz * dx);
}

#define ORC_BINS 16
#define ORC_LEAF 4

orc_bvh *orc_bvh_build(const float *tris, uint32_t n) {
    orc_bvh *b = (orc_bvh *)calloc(1, sizeof(orc_bvh));
    b->tris = tris;
    b->n = n;
    b->prims = (uint32_t *)malloc(sizeof(uint32_t) * (n ? n : 1));
    b->nodes = (orc_node *)malloc(sizeof(orc_node) * (2 * (size_t)(n ? n : 1)));
    if (n == 0) { b->n_nodes = 0; return b; }
    box3 *tb = (box3 *)malloc(sizeof(box3) * n);
    float *cen = (float *)malloc(sizeof(float) * 3 * n);
    for (uint32_t i = 0; i < n; ++i) {
        box_empty(&tb[i]);
        for (int k = 0; k < 3; ++k) box_grow_pt(&tb[i], tris + 9 * (size_t)i + 3 * k);
        for (int k = 0; k < 3; ++k) cen[3 * i + k] = 0.5f * (tb[i].bmin[k] + tb[i].bmax[k]);
        b->prims[i] = i;
    }
    /* explicit work stack: (node, first, count) */
    typedef struct { uint32_t node, first, count; } job;
    job *stack = (job *)malloc(sizeof(job) * 128);
    int sp = 0;
    b->n_nodes = 1;
    stack[sp++] = (job){0, 0, n};
    while (sp > 0) {
        job jb = stack[--sp];
        orc_node *nd = &b->nodes[jb.node];
        box3 nb, cb;
        box_empty(&nb); box_empty(&cb);
        for (uint32_t i = 0; i < jb.count; ++i) {
            uint32_t p = b->prims[jb.first + i];
            box_grow(&nb, &tb[p]);
            box_grow_pt(&cb, cen + 3 * p);
        }
        for (int k = 0; k < 3; ++k) { nd->bmin[k] = nb.bmin[k]; nd->bmax[k] = nb.bmax[k]; }
        int best_axis = -1, best_split = 0;
        float best_cost = FLT_MAX;
        if (jb.count > ORC_LEAF) {
            for (int ax = 0; ax < 3; ++ax) {
                float lo = cb.bmin[ax], hi = cb.bmax[ax];
                if (!(hi > lo)) continue;
                float scale = ORC_BINS / (hi - lo);
                box3 bins[ORC_BINS];
                uint32_t cnt[ORC_BINS] = {0};
                for (int i = 0; i < ORC_BINS; ++i) box_empty(&bins[i]);
                for (uint32_t i = 0; i < jb.count; ++i) {
                    uint32_t p = b->prims[jb.first + i];
                    int bi = (int)((cen[3 * p + ax] - lo) * scale);
                    if (bi >= ORC_BINS) bi = ORC_BINS - 1;
                    if (bi < 0) bi = 0;
                    cnt[bi]++;
                    box_grow(&bins[bi], &tb[p]);
                }
                float larea[ORC_BINS];
                uint32_t lcnt[ORC_BINS];
                box3 acc; box_empty(&acc); uint32_t c = 0;
                for (int i = 0; i < ORC_BINS; ++i) {
                    box_grow(&acc, &bins[i]); c += cnt[i];
                    larea[i] = box_area(&acc); lcnt[i] = c;
                }
                box_empty(&acc); c = 0;
                for (int i = ORC_BINS - 1; i > 0; --i) {
                    box_grow(&acc, &bins[i]); c += cnt[i];
                    float cost = larea[i - 1] * (float)lcnt[i - 1] + box_area(&acc) * (float)c;
                    if (lcnt[i - 1] > 0 && c > 0 && cost < best_cost) {
                        best_cost = cost; best_axis = ax; best_split = i;
                    }
                }
            }
        }
        if (best_axis < 0) {
            if (jb.count <= ORC_LEAF) {
                nd->left = (int32_t)jb.first; nd->count = (int32_t)jb.count;
                continue;
            }
            /* all centroids coincide: median split by index */
            best_axis = 0;
        }
        uint32_t mid;
        if (best_cost < FLT_MAX) {
            float lo = cb.bmin[best_axis], hi = cb.bmax[best_axis];
            float scale = ORC_BINS / (hi - lo);
            uint32_t i = jb.first, j = jb.first + jb.count;
            while (i < j) {
                uint32_t p = b->prims[i];
                int bi = (int)((cen[3 * p + best_axis] - lo) * scale);
                if (bi >= ORC_BINS) bi = ORC_BINS - 1;
                if (bi < 0) bi = 0;
                if (bi < best_split) ++i;
                else { --j; uint32_t t = b->prims[i]; b->prims[i] = b->prims[j]; b->prims[j] = t; }
            }
            mid = i;
        } else {
            mid = jb.first + jb.count / 2;
        }
        if (mid == jb.first || mid == jb.first + jb.count) mid = jb.first + jb.count / 2;
        uint32_t l = b->n_nodes;
        b->n_nodes += 2;
        nd->left = (int32_t)l; nd->count = 0;
        stack[sp++] = (job){l + 1, mid, jb.first + jb.count - mid};
        stack[sp++] = (job){l, jb.first, mid - jb.first};
        if (sp > 120) {
            /* deep degenerate input: grow the stack */
            job *ns = (job *)realloc(stack, sizeof(job) * (size_t)(sp * 2 + 128));
            stack = ns;
        }
    }
    free(stack);
    free(tb);
    free(cen);
    return b;
}

void orc_bvh_free(orc_bvh *b) {
    if (!b) return;
    free(b->nodes);
    free(b->prims);
    free(b);
}

uint32_t orc_bvh_node_count(const orc_bvh *b) { return b ? b->n_nodes : 0; }

/* Conservative slab test. Axes with a zero direction component only bound the origin. */
static int box_hit(const orc_node *nd, const orc_ray *r, float tfar_limit, float *tnear_out) {
    float tnear = r->tmin, tfar = tfar_limit;
    for (int i = 0; i < 3; ++i) {
        if (r->d[i] == 0.f) {
            if (r->o[i] < nd->bmin[i] || r->o[i] > nd->bmax[i]) return 0;
            continue;
        }
        float t0 = (nd->bmin[i] - r->o[i]) * r->inv_d[i];
        float t1 = (nd->bmax[i] - r->o[i]) * r->inv_d[i];
        if (t0 > t1) { float t = t0; t0 = t1; t1 = t; }
        t1 *= 1.f + 2.f * 1.7881393e-07f; /* 1 + 2*gamma(3), Ize 2013 */
        if (t0 > tnear) tnear = t0;
        if (t1 < tfar) tfar = t1;
    }
    *tnear_out = tnear;
    return tnear <= tfar;
}

static inline int better(float t, int32_t id, float best_t, int32_t best_id) {
    return t < best_t || (t == best_t && id < best_id);
}

/* closest hit; returns id or -1 */
int32_t orc_bvh_closest(const orc_bvh *b, const orc_ray *r, float *t, float *u, float *v,
                        uint64_t *nodes_visited, uint64_t *tris_tested) {
    int32_t best_id = -1;
    float best_t = r->tmax, bu = 0.f, bv = 0.f;
    if (!r->valid || b->n_nodes == 0) { *t = best_t; *u = 0.f; *v = 0.f; return -1; }
    uint32_t stack[256];
    int sp = 0;
    stack[sp++] = 0;
    uint64_t nv = 0, nt = 0;
    while (sp > 0) {
        uint32_t ni = stack[--sp];
        const orc_node *nd = &b->nodes[ni];
        float tn;
        ++nv;
        /* tie-inclusive culling: a triangle at exactly best_t with a lower id must survive */
        if (!box_hit(nd, r, best_t, &tn)) continue;
        if (nd->count > 0) {
            for (int32_t k = 0; k < nd->count; ++k) {
                uint32_t p = b->prims[nd->left + k];
                float tt, uu, vv;
                ++nt;
                if (orc_intersect_watertight(r, b->tris + 9 * (size_t)p, &tt, &uu, &vv) &&
                    tt < r->tmax && better(tt, (int32_t)p, best_t, best_id)) {
                    best_t = tt; best_id = (int32_t)p; bu = uu; bv = vv;
                }
            }
        } else {
            const orc_node *l = &b->nodes[nd->left], *rr = &b->nodes[nd->left + 1];
            float tl, tr;
            int hl = box_hit(l, r, best_t, &tl), hr = box_hit(rr, r, best_t, &tr);
            if (sp + 2 > 256) continue; /* cannot happen for SAH depth < 254 */
            if (hl && hr) {
                if (tl <= tr) { stack[sp++] = nd->left + 1; stack[sp++] = nd->left; }
                else { stack[sp++] = nd->left; stack[sp++] = nd->left + 1; }
            } else if (hl) stack[sp++] = nd->left;
            else if (hr) stack[sp++] = nd->left + 1;
        }
    }
    if (nodes_visited) *nodes_visited += nv;
    if (tris_tested) *tris_tested += nt;
    *t = best_t; *u = bu; *v = bv;
    return best_id;
}

/* ---------------------------------------------------------------- batch entry points */

typedef struct {
    const orc_bvh *bvh;
    const float *o, *d;
    fl_hit *hits;
    uint32_t begin, end;
    uint64_t nv, nt;
} trace_job;

static void *trace_worker(void *arg) {
    trace_job *j = (trace_job *)arg;
    for (uint32_t i = j->begin; i < j->end; ++i) {
        orc_ray r;
        orc_ray_precompute(j->o + 4 * (size_t)i, j->d + 4 * (size_t)i, &r);
        float t, u, v;
        int32_t id = orc_bvh_closest(j->bvh, &r, &t, &u, &v, &j->nv, &j->nt);
        j->hits[i].id = id;
        j->hits[i].t = id >= 0 ? t : r.tmax;
        j->hits[i].u = id >= 0 ? u : 0.f;
        j->hits[i].v = id >= 0 ? v : 0.f;
    }
    return NULL;
}

void orc_trace_closest(const orc_bvh *bvh, const float *org_tmin, const float *dir_tmax, uint32_t n,
                       fl_hit *hits, int nthreads, uint64_t *nodes_visited, uint64_t *tris_tested) {
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    pthread_t th[256];
    trace_job jobs[256];
    uint32_t chunk = (n + nthreads - 1) / nthreads;
    for (int k = 0; k < nthreads; ++k) {
        jobs[k].bvh = bvh; jobs[k].o = org_tmin; jobs[k].d = dir_tmax; jobs[k].hits = hits;
        jobs[k].begin = (uint32_t)((uint64_t)k * chunk < n ? (uint64_t)k * chunk : n);
        jobs[k].end = (uint32_t)((uint64_t)(k + 1) * chunk < n ? (uint64_t)(k + 1) * chunk : n);
        jobs[k].nv = jobs[k].nt = 0;
        pthread_create(&th[k], NULL, trace_worker, &jobs[k]);
    }
    uint64_t nv = 0, nt = 0;
    for (int k = 0; k < nthreads; ++k) {
        pthread_join(th[k], NULL);
        nv += jobs[k].nv; nt += jobs[k].nt;
    }
    if (nodes_visited) *nodes_visited = nv;
    if (tris_tested) *tris_tested = nt;
}

void orc_trace_brute(const float *tris, uint32_t n_tri, const float *org_tmin, const float *dir_tmax,
                     uint32_t n, fl_hit *hits) {
    for (uint32_t i = 0; i < n; ++i) {
        orc_ray r;
        orc_ray_precompute(org_tmin + 4 * (size_t)i, dir_tmax + 4 * (size_t)i, &r);
        int32_t best_id = -1;
        float best_t = r.tmax, bu = 0.f, bv = 0.f;
        if (r.valid) {
            for (uint32_t p = 0; p < n_tri; ++p) {
                float tt, uu, vv;
                if (orc_intersect_watertight(&r, tris + 9 * (size_t)p, &tt, &uu, &vv) && tt < r.tmax &&
                    better(tt, (int32_t)p, best_t, best_id)) {
                    best_t = tt; best_id = (int32_t)p; bu = uu; bv = vv;
                }
            }
        }
        hits[i].id = best_id;
        hits[i].t = best_t;
        hits[i].u = best_id >= 0 ? bu : 0.f;
        hits[i].v = best_id >= 0 ? bv : 0.f;
    }
}
