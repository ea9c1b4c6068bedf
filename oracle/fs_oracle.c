/* CPU oracle for the FARRSIGHT per-step hot path -- TEST INFRASTRUCTURE ONLY.
 * See fs_oracle.h for the pinning status of each part.  Built with
 * -ffp-contract=off so every expression rounds exactly as the reference's
 * g++ build (no fused multiply-adds on x86-64 without -mfma). */
#define _GNU_SOURCE
#include "fs_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* ======================================================================= */
/* Field: direct sum                                                        */
/* ======================================================================= */
/* src/FieldStructure.cpp:106-156.  Same expression order as the reference so
 * results agree bit for bit: per target a sequential sum over sources. */
void fso_direct_sum(double L, double eps, double* es, const double* targets, int nt,
                    const double* sources, const double* q_ws, int ns) {
    const double norm_const = 1 / sqrt(L * L + 4 * eps * eps);
#pragma omp parallel for schedule(static)
    for (int ii = 0; ii < nt; ++ii) {
        const double xi = targets[ii];
        double ei = 0.0;
        for (int jj = 0; jj < ns; ++jj) {
            double z = (xi - sources[jj]) / L;
            z = z - round(z);
            if (fabs(z - 0.5) < DBL_MIN || fabs(z + 0.5) < DBL_MIN || fabs(z) < DBL_MIN) continue;
            ei += q_ws[jj] * -1.0 * z * L * (norm_const - 1 / sqrt(4 * z * z * L * L + 4 * eps * eps));
        }
        es[ii] = ei;
    }
}

/* ======================================================================= */
/* Field: barycentric Lagrange treecode                                     */
/* ======================================================================= */
typedef struct {
    size_t m0, m1;          /* member range in permuted order (inclusive) */
    double x0, x1, xc;
    int nchild;
    int child[2];
} tc_node;

typedef struct {
    tc_node* nodes; int nnodes, cap;
    int* leaves; int nleaves, lcap;
    double* x; double* lam; int* old_index;
    double* tmpx; double* tmplam; int* tmpidx;
    size_t N0;
    int depth_guard;
} tc_tree;

static int tc_push(tc_tree* t, tc_node n) {
    if (t->nnodes == t->cap) {
        t->cap = t->cap ? 2 * t->cap : 64;
        t->nodes = (tc_node*)realloc(t->nodes, sizeof(tc_node) * t->cap);
    }
    t->nodes[t->nnodes] = n;
    return t->nnodes++;
}

/* split_2 (src/FieldStructure.cpp:547-630): stable partition of the node's
 * members into x <= midpoint and x > midpoint; children only when non-empty. */
static void tc_split(tc_tree* t, int ni) {
    tc_node nd = t->nodes[ni];
    const double mid = 0.5 * (nd.x0 + nd.x1);
    size_t start = nd.m0, end = nd.m1, k = 0;
    size_t nleft = 0;
    for (size_t i = start; i <= end; ++i)
        if (t->x[i] <= mid) nleft++;
    size_t li = 0, ri = nleft;
    for (size_t i = start; i <= end; ++i) {
        size_t dst = (t->x[i] <= mid) ? li++ : ri++;
        t->tmpx[dst] = t->x[i]; t->tmplam[dst] = t->lam[i]; t->tmpidx[dst] = t->old_index[i];
    }
    for (k = 0; k <= end - start; ++k) {
        t->x[start + k] = t->tmpx[k]; t->lam[start + k] = t->tmplam[k];
        t->old_index[start + k] = t->tmpidx[k];
    }
    size_t seg[2][2] = {{start, start + nleft - 1}, {start + nleft, end}};
    size_t cnt[2] = {nleft, end - start + 1 - nleft};
    for (int j = 0; j < 2; ++j) {
        if (cnt[j] == 0) continue;
        tc_node c;
        c.x0 = (j == 0) ? nd.x0 : mid;
        c.x1 = (j == 0) ? mid : nd.x1;
        c.xc = 0.5 * (c.x0 + c.x1);
        c.m0 = seg[j][0]; c.m1 = seg[j][1];
        c.nchild = 0;
        int ci = tc_push(t, c);
        t->nodes[ni].child[t->nodes[ni].nchild++] = ci;
    }
}

/* build_tree_1D_Recursive (src/FieldStructure.cpp:522-538). */
static int tc_build(tc_tree* t, int ni, int level) {
    if (level > 200) return -1;  /* the reference would recurse forever */
    size_t n = t->nodes[ni].m1 - t->nodes[ni].m0 + 1;
    if (n >= t->N0) {
        tc_split(t, ni);
        int nc = t->nodes[ni].nchild;
        for (int i = 0; i < nc; ++i)
            if (tc_build(t, t->nodes[ni].child[i], level + 1) < 0) return -1;
    } else {
        if (t->nleaves == t->lcap) {
            t->lcap = t->lcap ? 2 * t->lcap : 64;
            t->leaves = (int*)realloc(t->leaves, sizeof(int) * t->lcap);
        }
        t->leaves[t->nleaves++] = ni;
    }
    return 0;
}

typedef struct { int* v; int n, cap; } ivec;
static void ivec_push(ivec* a, int x) {
    if (a->n == a->cap) { a->cap = a->cap ? 2 * a->cap : 16; a->v = (int*)realloc(a->v, sizeof(int) * a->cap); }
    a->v[a->n++] = x;
}

/* build_interaction_list (src/FieldStructure.cpp:663-702). */
static void tc_lists(const tc_tree* t, double L, double sq_theta, int leaf_node, int pi,
                     ivec* far, ivec* near) {
    const tc_node* b = &t->nodes[leaf_node];
    const tc_node* p = &t->nodes[pi];
    double xcb = b->xc, xcp = p->xc, x_vb = b->x1, x_vp = p->x1;
    double r_dist = fabs(xcb - xcp);
    double dfbpx = fmin(r_dist, L - r_dist);
    double dfbx = x_vb - xcb;
    double dfpx = x_vp - xcp;
    double sq_R = dfbpx * dfbpx, sq_rb = dfbx * dfbx, sq_rp = dfpx * dfpx;
    if (p->nchild == 0) {
        ivec_push(near, pi);
    } else if ((sqrt(sq_rb) + sqrt(sq_rp)) / sqrt(sq_R) < sqrt(sq_theta)) {
        ivec_push(far, pi);
    } else {
        for (int i = 0; i < p->nchild; ++i) tc_lists(t, L, sq_theta, leaf_node, p->child[i], far, near);
    }
}

int fso_treecode(double L, double eps, double mac, int degree, int max_source, double* es,
                 const double* sources, const double* q_ws, int ns) {
    if (ns <= 0) return 0;
    const int P = degree, PP = P + 1;
    const double sq_theta = mac * mac;
    const double deno = L * L + 4 * eps * eps;
    const double pi = 3.14159265358979323846;
    tc_tree t;
    memset(&t, 0, sizeof(t));
    t.N0 = (size_t)max_source;
    t.x = (double*)malloc(sizeof(double) * ns);
    t.lam = (double*)malloc(sizeof(double) * ns);
    t.old_index = (int*)malloc(sizeof(int) * ns);
    t.tmpx = (double*)malloc(sizeof(double) * ns);
    t.tmplam = (double*)malloc(sizeof(double) * ns);
    t.tmpidx = (int*)malloc(sizeof(int) * ns);
    /* operator(): particles_x = fmod(src, L) (src/FieldStructure.cpp:235-247) */
    for (int i = 0; i < ns; ++i) { t.x[i] = fmod(sources[i], L); t.lam[i] = q_ws[i]; t.old_index[i] = i; }
    /* minval/maxval (src/FieldStructure.cpp:1032-1050) */
    double mn = t.x[0], mx = t.x[0];
    for (int i = 1; i < ns; ++i) { if (mn > t.x[i]) mn = t.x[i]; if (mx < t.x[i]) mx = t.x[i]; }
    tc_node root;
    root.m0 = 0; root.m1 = (size_t)ns - 1; root.x0 = mn - 0.1234; root.x1 = mx + 0.001;
    root.xc = 0.5 * (root.x0 + root.x1); root.nchild = 0;
    tc_push(&t, root);
    int rc = tc_build(&t, 0, 0);
    if (rc < 0) { es[0] = NAN; goto done; }
    {
        const int nnodes = t.nnodes;
        /* alloc_set_cluster_list (src/FieldStructure.cpp:775-866) */
        double* t1 = (double*)calloc((size_t)nnodes * PP, sizeof(double));
        double* mom = (double*)calloc((size_t)nnodes * PP, sizeof(double));
        double tch[64], w1i[64], dj[64], a1i[64];
        const double h = pi / P;
        for (int i = 0; i < PP; ++i) tch[i] = cos(i * h);
        dj[0] = 0.5; dj[P] = 0.5;
        for (int j = 1; j < P; ++j) dj[j] = 1.0;
        for (int j = 0; j < PP; ++j) w1i[j] = ((j % 2 == 0) ? 1 : -1) * dj[j];
        for (int ni = 1; ni < nnodes; ++ni) {
            const double x1 = t.nodes[ni].x0, x2 = t.nodes[ni].x1;
            double* tt = t1 + (size_t)ni * PP;
            double* mm = mom + (size_t)ni * PP;
            for (int j = 0; j < PP; ++j) tt[j] = x1 + (tch[j] + 1.0) * 0.5 * (x2 - x1);
            for (size_t k = t.nodes[ni].m0; k <= t.nodes[ni].m1; ++k) {
                const double x = t.x[k];
                int exact = -1;
                double sum = 0.0;
                for (int j = 0; j < PP; ++j) {
                    double dx = x - tt[j];
                    if (fabs(dx) <= DBL_MIN) exact = j;
                    else { a1i[j] = w1i[j] / dx; sum += a1i[j]; }
                }
                if (exact > -1) {
                    sum = 1.0;
                    for (int j = 0; j < PP; ++j) a1i[j] = 0.0;
                    a1i[exact] = 1.0;
                }
                const double D = 1.0 / sum;
                for (int i = 0; i < PP; ++i) { double s = a1i[i] * D; mm[i] += s * t.lam[k]; }
            }
        }
        /* interaction lists for every leaf */
        ivec* far = (ivec*)calloc(t.nleaves, sizeof(ivec));
        ivec* near = (ivec*)calloc(t.nleaves, sizeof(ivec));
        for (int l = 0; l < t.nleaves; ++l) tc_lists(&t, L, sq_theta, t.leaves[l], 0, &far[l], &near[l]);
        double* keps = (double*)calloc(ns, sizeof(double));
        /* Call_BL (src/FieldStructure.cpp:904-961) then Call_Ds (:963-1020) */
#pragma omp parallel for schedule(dynamic)
        for (int l = 0; l < t.nleaves; ++l) {
            const tc_node* lf = &t.nodes[t.leaves[l]];
            for (size_t ii = lf->m0; ii <= lf->m1; ++ii) {
                double tempx = 0.0;
                const double p_x = t.x[ii];
                for (int jj = 0; jj < far[l].n; ++jj) {
                    const int fi = far[l].v[jj];
                    for (int kk = 0; kk < PP; ++kk) {
                        double s = (p_x - t1[(size_t)fi * PP + kk]) / L;
                        s = s - round(s);
                        if (fabs(s - 0.5) < DBL_MIN || fabs(s + 0.5) < DBL_MIN || fabs(s) < DBL_MIN) continue;
                        tempx += mom[(size_t)fi * PP + kk] * -1.0 * s * (1 - sqrt(deno / (4 * s * s * L * L + 4 * eps * eps)));
                    }
                }
                keps[ii] += tempx;
            }
        }
#pragma omp parallel for schedule(dynamic)
        for (int l = 0; l < t.nleaves; ++l) {
            const tc_node* lf = &t.nodes[t.leaves[l]];
            for (size_t ii = lf->m0; ii <= lf->m1; ++ii) {
                double tempx = 0.0;
                for (int kk = 0; kk < near[l].n; ++kk) {
                    const tc_node* c = &t.nodes[near[l].v[kk]];
                    for (size_t jj = c->m0; jj <= c->m1; ++jj) {
                        double s = (t.x[ii] - t.x[jj]) / L;
                        s = s - round(s);
                        if (fabs(s - 0.5) < DBL_MIN || fabs(s + 0.5) < DBL_MIN || fabs(s) < DBL_MIN) continue;
                        tempx += t.lam[jj] * -1.0 * s * (1 - sqrt(deno / (4 * s * s * L * L + 4 * eps * eps)));
                    }
                }
                keps[ii] += tempx;
            }
        }
        /* back to the caller's order (src/FieldStructure.cpp:472-490) */
        for (int i = 0; i < ns; ++i) es[t.old_index[i]] = keps[i];
        rc = t.nleaves;
        for (int l = 0; l < t.nleaves; ++l) { free(far[l].v); free(near[l].v); }
        free(far); free(near); free(keps); free(t1); free(mom);
    }
done:
    free(t.nodes); free(t.leaves); free(t.x); free(t.lam); free(t.old_index);
    free(t.tmpx); free(t.tmplam); free(t.tmpidx);
    return rc;
}

/* ======================================================================= */
/* Panel mesh                                                               */
/* ======================================================================= */
typedef struct {
    int pts[9];
    int level, parent, which, child;
    int left, top, right, bottom;
    unsigned char lb, rb, xp, pr, needs;
} opanel;

struct fso_mesh {
    opanel* p; int np, pcap;
    double* xs; double* ps; int npts, xcap;
    int* leaves; int nleaves;
    int min_unrefined;
    int need_further;
    double xmin, xmax, pmin, pmax;
    int h, ph;
};

static int mesh_add_point(fso_mesh* m, double x, double p) {
    if (m->npts == m->xcap) {
        m->xcap = m->xcap ? 2 * m->xcap : 64;
        m->xs = (double*)realloc(m->xs, sizeof(double) * m->xcap);
        m->ps = (double*)realloc(m->ps, sizeof(double) * m->xcap);
    }
    m->xs[m->npts] = x; m->ps[m->npts] = p;
    return m->npts++;
}

static int mesh_add_panel(fso_mesh* m, opanel pn) {
    if (m->np == m->pcap) {
        m->pcap = m->pcap ? 2 * m->pcap : 64;
        m->p = (opanel*)realloc(m->p, sizeof(opanel) * m->pcap);
    }
    m->p[m->np] = pn;
    return m->np++;
}

static opanel mk_panel(int idx_unused, int level, int parent, int which, const int* pts,
                       int l, int t, int r, int b, int lb, int rb) {
    (void)idx_unused;
    opanel q;
    memset(&q, 0, sizeof(q));
    if (pts) memcpy(q.pts, pts, sizeof(q.pts));
    q.level = level; q.parent = parent; q.which = which; q.child = -1;
    q.left = l; q.top = t; q.right = r; q.bottom = b;
    q.lb = (unsigned char)lb; q.rb = (unsigned char)rb;
    return q;
}

/* refine_panels (src/structure_files/AMRStructure_amr.cpp:506-839), periodic,
 * non-adaptive.  Panel fields are read before any new panel is appended. */
static void mesh_refine_xp(fso_mesh* m) {
    const int nbefore = m->np;
    for (int jj = m->min_unrefined; jj < nbefore; ++jj) {
        if (!m->p[jj].needs) continue;
        const opanel P = m->p[jj];
        const double x0 = m->xs[P.pts[0]], p0 = m->ps[P.pts[0]];
        const double dx = m->xs[P.pts[3]] - x0;
        const double dp = m->ps[P.pts[1]] - p0;
        const double sdx = 0.5 * dx, sdp = 0.5 * dp;
        double sx[5], sp[5];
        for (int i = 0; i < 5; ++i) { sx[i] = x0 + sdx * i; sp[i] = p0 + sdp * i; }
        const int n = m->np;
        int p9, p10, p11, p18, p15, p22, p23, p24;
        int c0l = -1, c1l = -1, c0b = -1, c2b = -1, c1t = -1, c3t = -1, c2r = -1, c3r = -1;
        /* left edge */
        if (P.left == -2) {
            c0l = c1l = -2;
            p9 = mesh_add_point(m, sx[0], sp[1]); p10 = mesh_add_point(m, sx[0], sp[3]);
        } else if (P.left == -1) {
            opanel* pl = &m->p[m->p[P.parent].left];
            if (!pl->xp) { pl->needs = 1; m->need_further = 1; }
            p9 = mesh_add_point(m, sx[0], sp[1]); p10 = mesh_add_point(m, sx[0], sp[3]);
        } else if (!m->p[P.left].xp) {
            p9 = mesh_add_point(m, sx[0], sp[1]); p10 = mesh_add_point(m, sx[0], sp[3]);
        } else {
            c0l = m->p[P.left].child + 2; c1l = m->p[P.left].child + 3;
            m->p[c0l].right = n; m->p[c1l].right = n + 1;
            if (P.lb) { p9 = mesh_add_point(m, sx[0], sp[1]); p10 = mesh_add_point(m, sx[0], sp[3]); }
            else { p9 = m->p[c0l].pts[7]; p10 = m->p[c1l].pts[7]; }
        }
        /* bottom edge */
        if (P.bottom == -2) {
            c0b = c2b = -2;
            p11 = mesh_add_point(m, sx[1], sp[0]); p18 = mesh_add_point(m, sx[3], sp[0]);
        } else if (P.bottom == -1) {
            opanel* pb = &m->p[m->p[P.parent].bottom];
            if (!pb->xp) { pb->needs = 1; m->need_further = 1; }
            p11 = mesh_add_point(m, sx[1], sp[0]); p18 = mesh_add_point(m, sx[3], sp[0]);
        } else if (!m->p[P.bottom].xp) {
            p11 = mesh_add_point(m, sx[1], sp[0]); p18 = mesh_add_point(m, sx[3], sp[0]);
        } else {
            c0b = m->p[P.bottom].child + 1; c2b = m->p[P.bottom].child + 3;
            m->p[c0b].top = n; m->p[c2b].top = n + 2;
            p11 = m->p[c0b].pts[5]; p18 = m->p[c2b].pts[5];
        }
        /* top edge */
        if (P.top == -2) {
            c1t = c3t = -2;
            p15 = mesh_add_point(m, sx[1], sp[4]); p22 = mesh_add_point(m, sx[3], sp[4]);
        } else if (P.top == -1) {
            opanel* pt = &m->p[m->p[P.parent].top];
            if (!pt->xp) { pt->needs = 1; m->need_further = 1; }
            p15 = mesh_add_point(m, sx[1], sp[4]); p22 = mesh_add_point(m, sx[3], sp[4]);
        } else if (!m->p[P.top].xp) {
            p15 = mesh_add_point(m, sx[1], sp[4]); p22 = mesh_add_point(m, sx[3], sp[4]);
        } else {
            c1t = m->p[P.top].child; c3t = m->p[P.top].child + 2;
            m->p[c1t].bottom = n + 1; m->p[c3t].bottom = n + 3;
            p15 = m->p[c1t].pts[3]; p22 = m->p[c3t].pts[3];
        }
        /* right edge */
        if (P.right == -2) {
            c2r = c3r = -2;
            p23 = mesh_add_point(m, sx[4], sp[1]); p24 = mesh_add_point(m, sx[4], sp[3]);
        } else if (P.right == -1) {
            opanel* pr = &m->p[m->p[P.parent].right];
            if (!pr->xp) { pr->needs = 1; m->need_further = 1; }
            p23 = mesh_add_point(m, sx[4], sp[1]); p24 = mesh_add_point(m, sx[4], sp[3]);
        } else if (!m->p[P.right].xp) {
            p23 = mesh_add_point(m, sx[4], sp[1]); p24 = mesh_add_point(m, sx[4], sp[3]);
            if (P.right == jj) { c2r = n; c0l = n + 2; c3r = n + 1; c1l = n + 3; }
        } else {
            c2r = m->p[P.right].child; c3r = m->p[P.right].child + 1;
            m->p[c2r].left = n + 2; m->p[c3r].left = n + 3;
            if (P.rb) { p23 = mesh_add_point(m, sx[4], sp[1]); p24 = mesh_add_point(m, sx[4], sp[3]); }
            else { p23 = m->p[c2r].pts[1]; p24 = m->p[c3r].pts[1]; }
        }
        /* interior points: three on x1, two on x2, three on x3 */
        const int p12 = mesh_add_point(m, sx[1], sp[1]);
        mesh_add_point(m, sx[1], sp[2]); mesh_add_point(m, sx[1], sp[3]);
        const int p16 = mesh_add_point(m, sx[2], sp[1]);
        mesh_add_point(m, sx[2], sp[3]);
        const int p19 = mesh_add_point(m, sx[3], sp[1]);
        mesh_add_point(m, sx[3], sp[2]); mesh_add_point(m, sx[3], sp[3]);
        m->p[jj].xp = 1; m->p[jj].needs = 0; m->p[jj].child = n;
        const int* q = P.pts;
        int a[9] = {q[0], p9, q[1], p11, p12, p12 + 1, q[3], p16, q[4]};
        int b[9] = {q[1], p10, q[2], p12 + 1, p12 + 2, p15, q[4], p16 + 1, q[5]};
        int c[9] = {q[3], p16, q[4], p18, p19, p19 + 1, q[6], p23, q[7]};
        int d[9] = {q[4], p16 + 1, q[5], p19 + 1, p19 + 2, p22, q[7], p24, q[8]};
        const int lvl = P.level + 1;
        mesh_add_panel(m, mk_panel(n, lvl, jj, 0, a, c0l, n + 1, n + 2, c0b, P.lb, 0));
        mesh_add_panel(m, mk_panel(n + 1, lvl, jj, 1, b, c1l, c1t, n + 3, n, P.lb, 0));
        mesh_add_panel(m, mk_panel(n + 2, lvl, jj, 2, c, n, n + 3, c2r, c2b, 0, P.rb));
        mesh_add_panel(m, mk_panel(n + 3, lvl, jj, 3, d, n + 1, c3t, c3r, n + 2, 0, P.rb));
    }
}

/* refine_panels_refine_v (src/structure_files/AMRStructure_amr.cpp:233-504). */
static void mesh_refine_p(fso_mesh* m) {
    const int nbefore = m->np;
    for (int jj = m->min_unrefined; jj < nbefore; ++jj) {
        if (!m->p[jj].needs) continue;
        const opanel P = m->p[jj];
        const double x0 = m->xs[P.pts[0]], p0 = m->ps[P.pts[0]];
        const double dx = m->xs[P.pts[3]] - x0;
        const double dp = m->ps[P.pts[1]] - p0;
        const double sdp = 0.5 * dp, sdx = 0.5 * dx;
        double sx[5], sp[5];
        for (int i = 0; i < 5; ++i) { sp[i] = p0 + sdp * i; sx[i] = x0 + sdx * i; }
        const int n = m->np;
        int p9, p10, p13, p14;
        int c0b = -1, c0l = n, c0r = n, c1l = n + 1, c1t = -1, c1r = n + 1;
        if (P.left == -2) {
            c0l = c1l = -2;
            p9 = mesh_add_point(m, sx[0], sp[1]); p10 = mesh_add_point(m, sx[0], sp[3]);
        } else if (P.left == -1) {
            opanel* pl = &m->p[m->p[P.parent].left];
            if (!(pl->xp || pl->pr)) { pl->needs = 1; m->need_further = 1; }
            p9 = mesh_add_point(m, sx[0], sp[1]); p10 = mesh_add_point(m, sx[0], sp[3]);
        } else if (!(m->p[P.left].xp || m->p[P.left].pr)) {
            p9 = mesh_add_point(m, sx[0], sp[1]); p10 = mesh_add_point(m, sx[0], sp[3]);
        } else {
            const opanel* ln = &m->p[P.left];
            if (ln->xp) { c0l = ln->child + 2; c1l = ln->child + 3; }
            else { c0l = ln->child; c1l = ln->child + 1; }
            m->p[c0l].right = n; m->p[c1l].right = n + 1;
            if (P.lb) { p9 = mesh_add_point(m, sx[0], sp[1]); p10 = mesh_add_point(m, sx[0], sp[3]); }
            else { p9 = m->p[c0l].pts[7]; p10 = m->p[c1l].pts[7]; }
        }
        if (P.bottom == -2) {
            c0b = -2;
        } else if (P.bottom >= 0) {
            opanel* bn = &m->p[P.bottom];
            if (!bn->xp) {
                if (!bn->pr) { c0b = P.bottom; bn->top = n; }
                else { c0b = bn->child + 1; m->p[c0b].top = n; }
            }
        }
        if (P.top == -2) {
            c1t = -2;
        } else if (P.top >= 0) {
            const opanel* tn = &m->p[P.top];
            if (!tn->xp) {
                if (!tn->pr) c1t = -1;
                else { c1t = tn->child; m->p[c1t].bottom = n + 1; }
            }
        }
        if (P.right == -2) {
            c0r = c1r = -2;
            p13 = mesh_add_point(m, sx[4], sp[1]); p14 = mesh_add_point(m, sx[4], sp[3]);
        } else if (P.right == -1) {
            opanel* prn = &m->p[m->p[P.parent].right];
            if (!(prn->xp || prn->pr)) { prn->needs = 1; m->need_further = 1; }
            p13 = mesh_add_point(m, sx[4], sp[1]); p14 = mesh_add_point(m, sx[4], sp[3]);
        } else if (!(m->p[P.right].xp || m->p[P.right].pr)) {
            p13 = mesh_add_point(m, sx[4], sp[1]); p14 = mesh_add_point(m, sx[4], sp[3]);
        } else {
            const int rc = m->p[P.right].child;
            c0r = rc; c1r = rc + 1;
            m->p[c0r].left = n; m->p[c1r].left = n + 1;
            if (P.rb) { p13 = mesh_add_point(m, sx[4], sp[1]); p14 = mesh_add_point(m, sx[4], sp[3]); }
            else { p13 = m->p[c0r].pts[1]; p14 = m->p[c1r].pts[1]; }
        }
        const int p11 = mesh_add_point(m, sx[2], sp[1]);
        mesh_add_point(m, sx[2], sp[3]);
        m->p[jj].pr = 1; m->p[jj].needs = 0; m->p[jj].child = n;
        const int* q = P.pts;
        int a[9] = {q[0], p9, q[1], q[3], p11, q[4], q[6], p13, q[7]};
        int b[9] = {q[1], p10, q[2], q[4], p11 + 1, q[5], q[7], p14, q[8]};
        const int lvl = P.level + 1;
        mesh_add_panel(m, mk_panel(n, lvl, jj, 0, a, c0l, n + 1, c0r, c0b, P.lb, P.rb));
        mesh_add_panel(m, mk_panel(n + 1, lvl, jj, 1, b, c1l, c1t, c1r, n, P.lb, P.rb));
    }
}

static void mesh_collect_leaves(fso_mesh* m, int pi) {
    const opanel* P = &m->p[pi];
    if (P->pr) { for (int i = 0; i < 2; ++i) mesh_collect_leaves(m, P->child + i); }
    else if (P->xp) { for (int i = 0; i < 4; ++i) mesh_collect_leaves(m, P->child + i); }
    else m->leaves[m->nleaves++] = pi;
}

fso_mesh* fso_mesh_build(int h, int ph, double xmin, double xmax, double pmin, double pmax) {
    if (h < 1 || ph < 0) return NULL;
    fso_mesh* m = (fso_mesh*)calloc(1, sizeof(fso_mesh));
    m->xmin = xmin; m->xmax = xmax; m->pmin = pmin; m->pmax = pmax; m->h = h; m->ph = ph;
    /* create_prerefined_mesh (AMRStructure_amr.cpp:127-230) */
    const double dx = (xmax - xmin) / 4, dp = (pmax - pmin) / 4;
    double xi[5], pi_[5];
    for (int i = 0; i < 5; ++i) { xi[i] = xmin + i * dx; pi_[i] = pmin + i * dp; }
    for (int i = 0; i < 5; i += 2)
        for (int j = 0; j < 5; j += 2) mesh_add_point(m, xi[i], pi_[j]);
    for (int i = 0; i < 2; ++i) {
        mesh_add_point(m, xi[2 * i], pi_[1]); mesh_add_point(m, xi[2 * i], pi_[3]);
        for (int j = 0; j < 5; ++j) mesh_add_point(m, xi[1 + 2 * i], pi_[j]);
    }
    for (int j = 1; j < 5; j += 2) mesh_add_point(m, xi[4], pi_[j]);
    int root_pts[9] = {0, 1, 2, 3, 4, 5, 6, 7, 8};
    opanel root = mk_panel(0, 0, -1, -1, root_pts, 0, -2, 0, -2, 1, 1);
    mesh_add_panel(m, root);
    int a[9] = {0, 9, 1, 11, 12, 13, 3, 16, 4};
    int b[9] = {1, 10, 2, 13, 14, 15, 4, 17, 5};
    int c[9] = {3, 16, 4, 18, 19, 20, 6, 23, 7};
    int d[9] = {4, 17, 5, 20, 21, 22, 7, 24, 8};
    mesh_add_panel(m, mk_panel(1, 1, 0, 0, a, 3, 2, 3, -2, 1, 0));
    mesh_add_panel(m, mk_panel(2, 1, 0, 1, b, 4, -2, 4, 1, 1, 0));
    mesh_add_panel(m, mk_panel(3, 1, 0, 2, c, 1, 4, 1, -2, 0, 1));
    mesh_add_panel(m, mk_panel(4, 1, 0, 3, d, 2, -2, 2, 3, 0, 1));
    for (int i = 1; i <= 4; ++i) m->p[i].needs = 1;
    m->p[0].xp = 1; m->p[0].child = 1;
    m->min_unrefined = 1;
    for (int level = 1; level < h; ++level) {
        int npre = m->np;
        for (int i = m->min_unrefined; i < m->np; ++i) m->p[i].needs = 1;
        mesh_refine_xp(m);
        m->min_unrefined = npre;
    }
    for (int level = 0; level < ph; ++level) {
        int npre = m->np;
        for (int i = m->min_unrefined; i < m->np; ++i) m->p[i].needs = 1;
        mesh_refine_p(m);
        m->min_unrefined = npre;
    }
    m->leaves = (int*)malloc(sizeof(int) * m->np);
    m->nleaves = 0;
    mesh_collect_leaves(m, 0);
    return m;
}

void fso_mesh_destroy(fso_mesh* m) {
    if (!m) return;
    free(m->p); free(m->xs); free(m->ps); free(m->leaves); free(m);
}
int fso_mesh_npoints(const fso_mesh* m) { return m->npts; }
int fso_mesh_npanels(const fso_mesh* m) { return m->np; }
int fso_mesh_nleaves(const fso_mesh* m) { return m->nleaves; }
void fso_mesh_points(const fso_mesh* m, double* xs, double* ps) {
    memcpy(xs, m->xs, sizeof(double) * m->npts);
    memcpy(ps, m->ps, sizeof(double) * m->npts);
}
void fso_mesh_panels(const fso_mesh* m, int* rec) {
    for (int i = 0; i < m->np; ++i) {
        const opanel* P = &m->p[i];
        int* r = rec + (size_t)i * FSO_PANEL_INTS;
        for (int k = 0; k < 9; ++k) r[k] = P->pts[k];
        r[9] = P->level; r[10] = P->parent; r[11] = P->which; r[12] = P->child;
        r[13] = P->left; r[14] = P->top; r[15] = P->right; r[16] = P->bottom;
        r[17] = (P->lb ? 1 : 0) | (P->rb ? 2 : 0) | (P->xp ? 4 : 0) | (P->pr ? 8 : 0);
    }
}
void fso_mesh_leaves(const fso_mesh* m, int* leaf_inds) {
    memcpy(leaf_inds, m->leaves, sizeof(int) * m->nleaves);
}

/* recursively_set_leaves_weights (AMRStructure_amr.cpp:1102-1151) without *f. */
void fso_mesh_base_weights(const fso_mesh* m, double q, int quad, double* w) {
    memset(w, 0, sizeof(double) * m->npts);
    static const double wt[9] = {1.0, 2.0, 1.0, 2.0, 4.0, 2.0, 1.0, 2.0, 1.0};
    static const double ws[9] = {1.0, 4.0, 1.0, 4.0, 16.0, 4.0, 1.0, 4.0, 1.0};
    for (int l = 0; l < m->nleaves; ++l) {
        const opanel* P = &m->p[m->leaves[l]];
        double dx = m->xs[P->pts[3]] - m->xs[P->pts[0]];
        double p0 = m->ps[P->pts[0]], p1 = m->ps[P->pts[1]];
        double dp = p1 - p0;
        if (quad == 1) {
            double qdxdp9 = q * dx * dp / 9.0;
            for (int i = 0; i < 9; ++i) w[P->pts[i]] += qdxdp9 * ws[i];
        } else {
            double qdxdp4 = q * dx * dp / 4.0;
            for (int i = 0; i < 9; ++i) w[P->pts[i]] += qdxdp4 * wt[i];
        }
    }
}

/* ======================================================================= */
/* Initial conditions                                                       */
/* ======================================================================= */
static double f0_maxwell(double pth, double pstr, double p) {
    return 1.0 / sqrt(2.0 * M_PI) / pth * exp(-(p - pstr) * (p - pstr) / 2 / pth / pth);
}
double fso_f0(int ics, double pth, double pstr, double k, double amp, double x, double p) {
    switch (ics) {
    case 3: { /* F0_strong_two_stream: F0_LD(pth, k, amp)(x,p) * p * p */
        double ld = 1.0 / sqrt(2.0 * M_PI) / pth * exp(-(p - 0.0) * (p - 0.0) / 2 / pth / pth) * (1 + amp * cos(k * x));
        return ld * p * p;
    }
    case 4: /* F0_colder_two_stream */
        return .5 * (f0_maxwell(pth, 0.0, p - pstr) + f0_maxwell(pth, 0.0, p + pstr)) * (1 + amp * cos(k * x));
    case 1: case 2: case 9: case 10: default:
        /* F0_LD, F0_ion_acoustic_electron, F0_ion_acoustic_ion share this form */
        return 1.0 / sqrt(2.0 * M_PI) / pth * exp(-(p - pstr) * (p - pstr) / 2 / pth / pth) * (1 + amp * cos(k * x));
    }
}

/* ---- special functions of the relativistic initial conditions ---- */
double fso_bessel_k1(double x) {
    /* K_1(x) = exp(-x) int_0^inf exp(-x (cosh t - 1)) cosh t dt.  The integrand
     * is even in t and analytic in |Im t| < pi/2, so the trapezoid rule on the
     * half line converges like exp(-pi^2 / h); for large x the integrand is a
     * Gaussian of width 1/sqrt(x), whose error exp(-2 pi^2 / (h^2 x)) sets
     * h <= 0.25 / sqrt(x).  cosh t - 1 = 2 sinh^2(t/2) keeps the exponent
     * accurate near t = 0; the terms are added with Neumaier's compensated sum. */
    if (!(x > 0)) return NAN;
    const double h = fmin(1.0 / 16, 0.25 / sqrt(x));
    double sum = 0.5, comp = 0.0;
    for (int i = 1; i < 10000000; ++i) {
        const double t = i * h, sh = sinh(0.5 * t), ch = cosh(t);
        const double term = exp(-x * (2.0 * sh * sh)) * ch;
        const double y = sum + term;
        comp += fabs(sum) >= fabs(term) ? (sum - y) + term : (term - y) + sum;
        sum = y;
        if (term < 1e-20 * sum) break;
    }
    return exp(-x) * ((sum + comp) * h);
}

/* Carlson's R_F(x, y, z) and R_D(x, y, z): duplicate until every relative
 * deviation from the mean is below 2e-5, then the fifth-order series. */
static double carlson_rf(double x, double y, double z) {
    for (int it = 0; it < 200; ++it) {
        const double A = (x + y + z) / 3.0;
        const double X = 1.0 - x / A, Y = 1.0 - y / A, Z = 1.0 - z / A;
        if (fmax(fabs(X), fmax(fabs(Y), fabs(Z))) < 2e-5) {
            const double e2 = X * Y - Z * Z, e3 = X * Y * Z;
            return (1.0 - e2 / 10.0 + e3 / 14.0 + e2 * e2 / 24.0 - 3.0 * e2 * e3 / 44.0) / sqrt(A);
        }
        const double sx = sqrt(x), sy = sqrt(y), sz = sqrt(z);
        const double lam = sx * sy + sy * sz + sz * sx;
        x = 0.25 * (x + lam);
        y = 0.25 * (y + lam);
        z = 0.25 * (z + lam);
    }
    return NAN;
}
static double carlson_rd(double x, double y, double z) {
    double sum = 0.0, fac = 1.0;
    for (int it = 0; it < 200; ++it) {
        const double A = (x + y + 3.0 * z) / 5.0;
        const double X = 1.0 - x / A, Y = 1.0 - y / A, Z = 1.0 - z / A;
        if (fmax(fabs(X), fmax(fabs(Y), fabs(Z))) < 2e-5) {
            const double xy = X * Y, zz = Z * Z;
            const double e2 = xy - 6.0 * zz, e3 = (3.0 * xy - 8.0 * zz) * Z;
            const double e4 = 3.0 * (xy - zz) * zz, e5 = xy * zz * Z;
            const double ser = 1.0 - 3.0 * e2 / 14.0 + e3 / 6.0 + 9.0 * e2 * e2 / 88.0 - 3.0 * e4 / 22.0
                             - 9.0 * e2 * e3 / 52.0 + 3.0 * e5 / 26.0;
            return 3.0 * sum + fac * ser / (A * sqrt(A));
        }
        const double sx = sqrt(x), sy = sqrt(y), sz = sqrt(z);
        const double lam = sx * sy + sy * sz + sz * sx;
        sum += fac / (sz * (z + lam));
        fac *= 0.25;
        x = 0.25 * (x + lam);
        y = 0.25 * (y + lam);
        z = 0.25 * (z + lam);
    }
    return NAN;
}
/* phi reduced to [-pi/2, pi/2] plus n half periods */
static double ell_reduce(double phi, double* n) {
    *n = floor(phi / M_PI + 0.5);
    return phi - *n * M_PI;
}
double fso_ellint_1(double k, double phi) {
    double n;
    const double r = ell_reduce(phi, &n), s = sin(r), c = cos(r);
    double v = s * carlson_rf(c * c, 1.0 - k * k * s * s, 1.0);
    if (n != 0) v += 2.0 * n * carlson_rf(0.0, 1.0 - k * k, 1.0);
    return v;
}
double fso_ellint_2(double k, double phi) {
    double n;
    const double r = ell_reduce(phi, &n), s = sin(r), c = cos(r), kk = k * k, y = 1.0 - kk * s * s;
    double v = s * carlson_rf(c * c, y, 1.0) - kk * s * s * s * carlson_rd(c * c, y, 1.0) / 3.0;
    if (n != 0)
        v += 2.0 * n * (carlson_rf(0.0, 1.0 - kk, 1.0) - kk * carlson_rd(0.0, 1.0 - kk, 1.0) / 3.0);
    return v;
}

/* ---- make_f0_return_ptr (AMRSimulation_load.cpp:139-225) ---- */
#define FSO_WAVE_NODES 100
struct fso_dist {
    int ics;
    double pth, pstr, amp, k, mu;
    /* F0_Friedman_beam (initial_distributions.cpp:171-184, 241-290) */
    double fb_xcf, fb_nhat, fb_pth, fb_dx;
    int fb_n;
    double* fb_N;
    /* Maxwell_Jutner / Relativistic_Two_Stream (:306-313, :350-360) */
    double k1mu, gstr;
    /* Relativistic_Wave (:366-452) */
    double wv_x[FSO_WAVE_NODES], wv_p[FSO_WAVE_NODES];
};

fso_dist* fso_dist_create(const fso_species_params* q, double xmin, double xmax, int* rc) {
    *rc = 0;
    fso_dist* d = (fso_dist*)calloc(1, sizeof(fso_dist));
    d->ics = q->ics_type;
    d->pth = q->pth; d->pstr = q->pstr; d->amp = q->amp; d->mu = q->mu;
    d->k = 2.0 * M_PI / (xmax - xmin) * q->normalized_wavenumber;  /* kx of make_f0_return_ptr */
    if (d->ics == 5) {
        /* Delta = amp, Tstar = pth^2, xmax = the deck's xmax; the envelope
         * N'' = N^2 - (1 + Delta) N + N'^2 / N, N(0) = 1, N'(0) = 0, by explicit
         * Euler with step 0.01 out to 1.1 xmax in units of gamma_b lambda_D */
        const double kb0 = 2.0 * M_PI / 3.0, lamD = 2.81e-4, bb = 2.343e-3;
        const double gb = 1.0 / sqrt(1 + bb * bb);
        const double dx = 0.01;
        d->fb_xcf = 1.0 / kb0 / lamD / gb;
        d->fb_nhat = 1.0 / (1.0 + d->amp);
        d->fb_pth = sqrt(q->pth * q->pth);
        const double nxd = ceil(1.1 * (xmax * d->fb_xcf) / dx);
        if (!(nxd >= 2) || nxd > 1e8) { *rc = 1; fso_dist_destroy(d); return NULL; }
        d->fb_n = (int)nxd;
        d->fb_N = (double*)calloc((size_t)d->fb_n, sizeof(double));
        d->fb_N[0] = 1.0;
        double dN = 0.0;
        for (int i = 1; i < d->fb_n; ++i) {
            const double n0 = d->fb_N[i - 1];
            if (n0 <= 1e-150) continue;  /* density below the floor stays 0 */
            d->fb_N[i] = n0 + dx * dN;
            dN += dx * (n0 * n0 - n0 * (1 + d->amp) + 1.0 / n0 * dN * dN);
        }
        d->fb_dx = 1 * dx - 0.0;
    } else if (d->ics == 6 || d->ics == 7) {
        if (!(d->mu > 0)) { *rc = 1; fso_dist_destroy(d); return NULL; }
        d->k1mu = fso_bessel_k1(d->mu);
        if (!(d->k1mu > 0) || !isfinite(d->k1mu)) { *rc = 1; fso_dist_destroy(d); return NULL; }
        d->gstr = sqrt(1 + d->pstr * d->pstr);
    } else if (d->ics == 8) {
        /* cold orbit of a wave with maximum gamma gm = amp and phase velocity
         * wave_beta, sampled at 100 values of the orbit parameter alpha in
         * [-pi/2, 5 pi/2] */
        const double gm = d->amp, wb = q->wave_beta;
        if (!(gm >= 1) || (wb < 1.0 && 1.0 / sqrt(1 - wb * wb) < gm)) { *rc = 1; fso_dist_destroy(d); return NULL; }
        const double kap = sqrt((gm - 1.0) / (gm + 1.0)), kp = sqrt(2 / (gm + 1.0));
        const double da = 3 * M_PI / (FSO_WAVE_NODES - 1);
        for (int i = 0; i < FSO_WAVE_NODES; ++i) {
            const double a = -M_PI / 2 + i * da;
            const double x0 = wb * (2 / kp * fso_ellint_2(kap, a) - kp * fso_ellint_1(kap, a));
            d->wv_x[i] = x0 + 2 * kap / kp * sin(a);
            const double g = gm - (gm - 1) * sin(a) * sin(a);
            d->wv_p[i] = sqrt(g * g - 1) * (cos(a) > 0 ? 1 : -1);
        }
    }
    return d;
}

double fso_dist_eval(const fso_dist* d, double x, double p, int* rc) {
    const double c = 1.0 / sqrt(2.0 * M_PI);
    switch (d->ics) {
    case 5: {
        const double pp = p * 1.25;  /* maxwellian(x, p mu) nhat N(x / mu), mu = 1.25 */
        const double m = c / d->fb_pth * exp(-(pp - 0.0) * (pp - 0.0) / 2 / d->fb_pth / d->fb_pth);
        const double u = fabs(x / 1.25) * d->fb_xcf / d->fb_dx;
        const double fl = floor(u);
        if (!(fl >= 0) || fl + 1 >= (double)d->fb_n) { *rc = 1; return 0.0; }
        const int i = (int)fl;
        const double th = u - fl;
        return m * d->fb_nhat * ((1 - th) * d->fb_N[i] + th * d->fb_N[i + 1]);
    }
    case 6: {
        const double g = sqrt(1 + p * p);
        return exp(-g * d->mu) / 2.0 / d->k1mu * (1 + d->amp * cos(d->k * x));
    }
    case 7: {
        const double g = sqrt(1 + p * p), ppm = p * d->pstr * d->mu;
        const double ep = exp(ppm - d->gstr * g * d->mu) / 2.0 / d->k1mu;
        const double em = exp(-ppm - d->gstr * g * d->mu) / 2.0 / d->k1mu;
        return (ep + em) / 2.0 * (1 + d->amp * cos(d->k * x));
    }
    case 8: {
        if (!(x <= d->wv_x[FSO_WAVE_NODES - 1])) { *rc = 1; return 0.0; }
        int i = 0;
        while (x > d->wv_x[i + 1]) ++i;
        const double th = x - d->wv_x[i];  /* offset from the node, not normalised */
        const double p0 = (1 - th) * d->wv_p[i] + th * d->wv_p[i + 1];
        return 1.0 / sqrt(2 * M_PI) / d->pth * exp(-(p - p0) * (p - p0) / 2 / d->pth / d->pth);
    }
    default:
        return fso_f0(d->ics, d->pth, d->pstr, d->k, d->amp, x, p);
    }
}

void fso_dist_destroy(fso_dist* d) {
    if (!d) return;
    free(d->fb_N);
    free(d);
}

/* ======================================================================= */
/* Remesh: point location and 9-point fit                                   */
/* ======================================================================= */
typedef struct {
    const fso_mesh* m;
    const double* ox; const double* op;
    double Lx;
} locate_ctx;

/* find_leaf_containing_point_from_neighbor (AMRStructure_interp.cpp:12-230),
 * written as a loop: tx is updated in place, beyond_boundary is or-ed over every
 * visited panel, the walk stops at the first revisited panel. */
static int walk_from(const locate_ctx* c, double* tx, double tp, int* beyond, int leaf,
                     int* hist, int* nhist, int hcap) {
    const opanel* pn = c->m->p;
    const double Lx = c->Lx;
    for (;;) {
        if (leaf == 0) {
            if (*nhist < hcap) hist[(*nhist)++] = 0;
            return 0;
        }
        const opanel* P = &pn[leaf];
        const double x_bl = c->ox[P->pts[0]], p_bl = c->op[P->pts[0]];
        const double x_tl = c->ox[P->pts[2]], p_tl = c->op[P->pts[2]];
        const double x_mid = c->ox[P->pts[4]];
        const double x_br = c->ox[P->pts[6]], p_br = c->op[P->pts[6]];
        const double x_tr = c->ox[P->pts[8]], p_tr = c->op[P->pts[8]];
        if (*tx - x_mid >= Lx / 2) *tx -= Lx;
        if (*tx - x_mid < -Lx / 2) *tx += Lx;
        const double t = *tx;
        int ir = (x_tr - x_br) * (tp - p_br) > (p_tr - p_br) * (t - (x_br));
        int il = (x_tl - x_bl) * (tp - p_bl) <= (p_tl - p_bl) * (t - x_bl);
        int it = (x_tr - x_tl) * (tp - p_tl) < (p_tr - p_tl) * (t - x_tl);
        int ib = (x_br - x_bl) * (tp - p_bl) >= (p_br - p_bl) * (t - x_bl);
        int nl = leaf;
        if (!ir && P->right != -2) {
            if (P->rb) *tx -= Lx;
            if (P->right == -1) nl = pn[P->parent].right;
            else nl = pn[P->right].xp ? pn[P->right].child : P->right;
        } else if (!it && P->top != -2) {
            if (P->top == -1) nl = pn[P->parent].top;
            else nl = pn[P->top].xp ? pn[P->top].child : P->top;
        } else if (!ib && P->bottom != -2) {
            if (P->bottom == -1) nl = pn[P->parent].bottom;
            else nl = pn[P->bottom].xp ? pn[P->bottom].child + 1 : P->bottom;
        } else if (!il && P->left != -2) {
            if (P->lb) *tx += Lx;
            if (P->left == -1) nl = pn[P->parent].left;
            else nl = pn[P->left].xp ? pn[P->left].child + 2 : P->left;
        }
        if ((!ir && P->right == -2) || (!il && P->left == -2) || (!it && P->top == -2) ||
            (!ib && P->bottom == -2))
            *beyond = 1;
        int seen = 0;
        for (int i = 0; i < *nhist; ++i) if (hist[i] == nl) { seen = 1; break; }
        if (seen || *nhist >= hcap) return nl;
        hist[(*nhist)++] = nl;
        leaf = nl;
    }
}

/* find_leaf_containing_xp_recursively (AMRStructure_interp.cpp:232-426). */
static int find_recursive(const locate_ctx* c, double* x, double p, int* beyond, int pi) {
    const opanel* pn = c->m->p;
    const double Lx = c->Lx;
    for (;;) {
        const opanel* P = &pn[pi];
        const int cs = P->child;
        if (!(P->xp || P->pr)) {
            const double x_bl = c->ox[P->pts[0]], p_bl = c->op[P->pts[0]];
            const double x_tl = c->ox[P->pts[2]], p_tl = c->op[P->pts[2]];
            const double x_br = c->ox[P->pts[6]], p_br = c->op[P->pts[6]];
            const double x_tr = c->ox[P->pts[8]], p_tr = c->op[P->pts[8]];
            const double X = *x;
            int ir = (x_tr - x_br) * (p - p_br) > (p_tr - p_br) * (X - (x_br));
            int il = (x_tl - x_bl) * (p - p_bl) <= (p_tl - p_bl) * (X - x_bl);
            int it = (x_tr - x_tl) * (p - p_tl) < (p_tr - p_tl) * (X - x_tl);
            int ib = (x_br - x_bl) * (p - p_bl) >= (p_br - p_bl) * (X - x_bl);
            if ((!il && P->left == -2) || (!ir && P->right == -2) || (!it && P->top == -2) ||
                (!ib && P->bottom == -2))
                *beyond = 1;
            return pi;
        }
        double X = *x;
        const double x_bl = c->ox[P->pts[0]], p_bl = c->op[P->pts[0]];
        const double x_ml = c->ox[P->pts[1]], p_ml = c->op[P->pts[1]];
        const double x_tl = c->ox[P->pts[2]], p_tl = c->op[P->pts[2]];
        const double x_bm = c->ox[P->pts[3]], p_bm = c->op[P->pts[3]];
        const double x_mm = c->ox[P->pts[4]], p_mm = c->op[P->pts[4]];
        const double x_tm = c->ox[P->pts[5]], p_tm = c->op[P->pts[5]];
        const double x_br = c->ox[P->pts[6]], p_br = c->op[P->pts[6]];
        const double x_mr = c->ox[P->pts[7]], p_mr = c->op[P->pts[7]];
        const double x_tr = c->ox[P->pts[8]], p_tr = c->op[P->pts[8]];
        int i1b = (x_mm - x_ml) * (p - p_ml) >= (p_mm - p_ml) * (X - x_ml);
        int i1r = (x_tm - x_mm) * (p - p_mm) >= (p_tm - p_mm) * (X - x_mm);
        int i3b = (x_mr - x_mm) * (p - p_mm) >= (p_mr - p_mm) * (X - x_mm);
        int sub;
        if (i1b && i1r) {
            int i1t = (x_tm - x_tl) * (p - p_tl) <= (p_tm - p_tl) * (X - x_tl);
            const opanel* c1 = &pn[cs + 1];
            if (i1t || c1->top < 0) {
                int i1l = (x_tl - x_ml) * (p - p_ml) <= (p_tl - p_ml) * (X - x_ml);
                if (i1l || c1->left < 0) sub = cs + 1;
                else { sub = c1->left; if (P->lb) *x += Lx; }
            } else sub = c1->top;
        } else if (i3b && !i1r) {
            int i3t = (x_tr - x_tm) * (p - p_tm) <= (p_tr - p_tm) * (X - x_tm);
            const opanel* c3 = P->pr ? &pn[cs + 1] : &pn[cs + 3];
            if (i3t || c3->top < 0) {
                int i3r = (x_tr - x_mr) * (p - p_mr) <= (p_tr - p_mr) * (X - x_mr);
                if (!i3r || c3->right < 0) sub = P->pr ? cs + 1 : cs + 3;
                else { sub = c3->right; if (P->rb) *x -= Lx; }
            } else sub = c3->top;
        } else {
            int i0r = (x_mm - x_bm) * (p - p_bm) >= (p_mm - p_bm) * (X - x_bm);
            if (i0r) {
                int i0b = (x_bm - x_bl) * (p - p_bl) >= (p_bm - p_bl) * (X - x_bl);
                const opanel* c0 = &pn[cs];
                if (i0b || c0->bottom < 0) {
                    int i0l = (x_ml - x_bl) * (p - p_bl) <= (p_ml - p_bl) * (X - x_bl);
                    if (i0l || c0->left < 0) sub = cs;
                    else { sub = c0->left; if (P->lb) *x += Lx; }
                } else sub = c0->bottom;
            } else {
                int i2b = (x_br - x_bm) * (p - p_bm) >= (p_br - p_bm) * (X - x_bm);
                const opanel* c2 = P->pr ? &pn[cs] : &pn[cs + 2];
                if (i2b || c2->bottom < 0) {
                    int i2r = (x_mr - x_br) * (p - p_br) <= (p_mr - p_br) * (X - x_br);
                    if (!i2r || c2->right < 0) sub = P->pr ? cs : cs + 2;
                    else { sub = c2->right; if (P->rb) *x -= Lx; }
                } else sub = c2->bottom;
            }
        }
        pi = sub;
    }
}

/* 9x9 solve with row pivoting by the largest |a| (first index on ties), the
 * algorithm class of Eigen's PartialPivLU used at AMRStructure_interp.cpp:935. */
static void lu_solve9(double A[9][9], double b[9]) {
    int perm[9];
    for (int i = 0; i < 9; ++i) perm[i] = i;
    for (int k = 0; k < 9; ++k) {
        int piv = k;
        double best = fabs(A[k][k]);
        for (int i = k + 1; i < 9; ++i) { double v = fabs(A[i][k]); if (v > best) { best = v; piv = i; } }
        if (piv != k) {
            for (int j = 0; j < 9; ++j) { double t = A[k][j]; A[k][j] = A[piv][j]; A[piv][j] = t; }
            int t = perm[k]; perm[k] = perm[piv]; perm[piv] = t;
        }
        if (best != 0.0)
            for (int i = k + 1; i < 9; ++i) A[i][k] = A[i][k] / A[k][k];
        for (int i = k + 1; i < 9; ++i)
            for (int j = k + 1; j < 9; ++j) A[i][j] = A[i][j] - A[i][k] * A[k][j];
    }
    double y[9];
    for (int i = 0; i < 9; ++i) y[i] = b[perm[i]];
    /* unit lower, column oriented */
    for (int k = 0; k < 9; ++k)
        for (int i = k + 1; i < 9; ++i) y[i] = y[i] - y[k] * A[i][k];
    /* upper, column oriented from the bottom */
    for (int k = 8; k >= 0; --k) {
        y[k] = y[k] / A[k][k];
        for (int i = 0; i < k; ++i) y[i] = y[i] - y[k] * A[i][k];
    }
    for (int i = 0; i < 9; ++i) b[i] = y[i];
}

/* interpolate_from_panel_to_points (AMRStructure_interp.cpp:795-975): fit the
 * 9 values of a panel in the monomial basis
 * {1, dx, dx dp, dp, dx^2, dx^2 dp, dx^2 dp^2, dx dp^2, dp^2} about point 4 and
 * evaluate it at each requested point. */
void fso_panel_fit(const double* px, const double* pp, const double* pf, int npts,
                   const double* x, const double* p, double* out) {
    double A[9][9], c[9], pdx[9], pdp[9];
    for (int i = 0; i < 9; ++i) { pdx[i] = px[i] - px[4]; pdp[i] = pp[i] - pp[4]; }
    for (int i = 0; i < 9; ++i) {
        A[i][0] = 1; A[i][1] = pdx[i];
        A[i][2] = pdx[i] * pdp[i];
        A[i][3] = pdp[i];
        A[i][4] = pdx[i] * pdx[i];
        A[i][5] = pdx[i] * pdx[i] * pdp[i];
        A[i][6] = pdx[i] * pdx[i] * pdp[i] * pdp[i];
        A[i][7] = pdx[i] * pdp[i] * pdp[i];
        A[i][8] = pdp[i] * pdp[i];
        c[i] = pf[i];
    }
    lu_solve9(A, c);
    for (int k = 0; k < npts; ++k) {
        double dx = x[k] - px[4], dp = p[k] - pp[4];
        double dxsq = dx * dx, dpsq = dp * dp;
        double D[9] = {1, dx, dx * dp, dp, dxsq, dxsq * dp, dxsq * dpsq, dx * dpsq, dpsq};
        double v = 0.0;
        for (int j = 0; j < 9; ++j) v += D[j] * c[j];
        out[k] = v;
    }
}

typedef struct { const double* sx; const double* sp; double thr; } sort_ctx;
static sort_ctx g_sort;
static int less_pt(int a, int b) {
    if (fabs(g_sort.sp[a] - g_sort.sp[b]) >= g_sort.thr) return g_sort.sp[a] < g_sort.sp[b];
    return g_sort.sx[a] < g_sort.sx[b];
}
static void merge_sort(int* v, int* tmp, int n) {
    if (n < 2) return;
    int h = n / 2;
    merge_sort(v, tmp, h);
    merge_sort(v + h, tmp, n - h);
    int i = 0, j = h, k = 0;
    while (i < h && j < n) tmp[k++] = less_pt(v[j], v[i]) ? v[j++] : v[i++];
    while (i < h) tmp[k++] = v[i++];
    while (j < n) tmp[k++] = v[j++];
    memcpy(v, tmp, sizeof(int) * n);
}

static int remesh_interp_impl(const fso_mesh* old_m, const fso_mesh* m, const double* old_xs,
                              const double* old_ps, const double* old_fs, double f_beyond, double* new_fs,
                              int* leaf_of_point, double* final_x);

int fso_remesh_interp(const fso_mesh* m, const double* old_xs, const double* old_ps,
                      const double* old_fs, double f_beyond, double* new_fs,
                      int* leaf_of_point, double* final_x) {
    return remesh_interp_impl(m, m, old_xs, old_ps, old_fs, f_beyond, new_fs, leaf_of_point, final_x);
}

int fso_remesh_interp2(const fso_mesh* old_m, const fso_mesh* new_m, const double* old_xs, const double* old_ps,
                       const double* old_fs, double f_beyond, double* new_fs) {
    return remesh_interp_impl(old_m, new_m, old_xs, old_ps, old_fs, f_beyond, new_fs, NULL, NULL);
}

/* old_m: panels of the previous mesh (positions old_xs/old_ps); m: the new
 * uniform mesh whose points are located. */
static int remesh_interp_impl(const fso_mesh* old_m, const fso_mesh* m, const double* old_xs,
                              const double* old_ps, const double* old_fs, double f_beyond, double* new_fs,
                              int* leaf_of_point, double* final_x) {
    const int N = m->npts;
    const double Lx = m->xmax - m->xmin;
    const int npx = 1 << m->h, npp = 1 << (m->h + m->ph);
    const int nx = 2 * npx + 1, np = 2 * npp + 1;
    const double initial_dp = (m->pmax - m->pmin) / npp;
    locate_ctx c = {old_m, old_xs, old_ps, Lx};
    /* shift_xs (AMRStructure_interp.cpp:429-491) */
    double* sx = (double*)malloc(sizeof(double) * N);
    const double x_bl = old_xs[0], p_bl = old_ps[0], x_tl = old_xs[2], p_tl = old_ps[2];
    const double x_br = old_xs[6], p_br = old_ps[6], x_tr = old_xs[8], p_tr = old_ps[8];
    int rc = 0;
    for (int i = 0; i < N; ++i) {
        double p = m->ps[i], xt = m->xs[i];
        int cnt = 0;
        while (!((x_tl - x_bl) * (p - p_bl) <= (p_tl - p_bl) * (xt - x_bl))) {
            xt += Lx;
            if (++cnt > 10) { rc = -1; break; }
        }
        cnt = 0;
        while (rc == 0 && !((x_tr - x_br) * (p - p_br) > (p_tr - p_br) * (xt - (x_br)))) {
            xt -= Lx;
            if (++cnt > 10) { rc = -1; break; }
        }
        if (rc) { free(sx); return rc; }
        sx[i] = xt;
    }
    /* sort by p row (threshold initial_dp/10) then shifted x (:525-558) */
    int* order = (int*)malloc(sizeof(int) * N);
    int* tmp = (int*)malloc(sizeof(int) * N);
    for (int i = 0; i < N; ++i) order[i] = i;
    g_sort.sx = sx; g_sort.sp = m->ps; g_sort.thr = initial_dp / 10.0;
    merge_sort(order, tmp, N);
    free(tmp);
    double* sortx = (double*)malloc(sizeof(double) * N);
    double* sortp = (double*)malloc(sizeof(double) * N);
    for (int i = 0; i < N; ++i) { sortx[i] = sx[order[i]]; sortp[i] = m->ps[order[i]]; }
    int* leaf = (int*)malloc(sizeof(int) * N);
    const int hcap = 1 << 16;
    int* hist = (int*)malloc(sizeof(int) * hcap);
    int beyond = 0;
    int leaf_ind = find_recursive(&c, &sortx[0], sortp[0], &beyond, 0);
    int* first_col = (int*)malloc(sizeof(int) * np);
    for (int ii = 0; ii < np; ++ii) {
        beyond = 0;
        int pt = ii * nx;
        int nh = 0;
        hist[nh++] = leaf_ind;
        leaf_ind = walk_from(&c, &sortx[pt], sortp[pt], &beyond, leaf_ind, hist, &nh, hcap);
        first_col[ii] = leaf_ind;
        leaf[pt] = beyond ? 0 : leaf_ind;
    }
    for (int ii = 0; ii < np; ++ii) {
        int pt = ii * nx;
        int lc = first_col[ii];
        for (int jj = 1; jj < nx; ++jj) {
            beyond = 0;
            pt++;
            int nh = 0;
            hist[nh++] = lc;
            lc = walk_from(&c, &sortx[pt], sortp[pt], &beyond, lc, hist, &nh, hcap);
            leaf[pt] = beyond ? 0 : lc;
        }
    }
    free(hist); free(first_col);
    /* per-panel fit, evaluated point by point */
    for (int k = 0; k < N; ++k) {
        double v;
        const int l = leaf[k];
        if (l == 0) v = f_beyond;
        else {
            const opanel* P = &old_m->p[l];
            double px[9], pp[9], pf[9];
            for (int i = 0; i < 9; ++i) { px[i] = old_xs[P->pts[i]]; pp[i] = old_ps[P->pts[i]]; pf[i] = old_fs[P->pts[i]]; }
            fso_panel_fit(px, pp, pf, 1, &sortx[k], &sortp[k], &v);
        }
        new_fs[order[k]] = v;
        if (leaf_of_point) leaf_of_point[order[k]] = l;
        if (final_x) final_x[order[k]] = sortx[k];
    }
    free(sx); free(order); free(sortx); free(sortp); free(leaf);
    return 0;
}

/* ======================================================================= */
/* Adaptive refinement                                                      */
/* ======================================================================= */
/* 9-point fit coefficients (the same LU as fso_panel_fit). */
static void fit_coefs(const double* px, const double* pp, const double* pf, double* c) {
    double A[9][9], pdx[9], pdp[9];
    for (int i = 0; i < 9; ++i) { pdx[i] = px[i] - px[4]; pdp[i] = pp[i] - pp[4]; }
    for (int i = 0; i < 9; ++i) {
        A[i][0] = 1; A[i][1] = pdx[i];
        A[i][2] = pdx[i] * pdp[i];
        A[i][3] = pdp[i];
        A[i][4] = pdx[i] * pdx[i];
        A[i][5] = pdx[i] * pdx[i] * pdp[i];
        A[i][6] = pdx[i] * pdx[i] * pdp[i] * pdp[i];
        A[i][7] = pdx[i] * pdp[i] * pdp[i];
        A[i][8] = pdp[i] * pdp[i];
        c[i] = pf[i];
    }
    lu_solve9(A, c);
}

double fso_interp_point(const fso_mesh* old_m, const double* old_xs, const double* old_ps, const double* old_fs,
                        double f_beyond, double x, double p, int* rc) {
    const double Lx = old_m->xmax - old_m->xmin;
    /* shift_xs for one point (:429-491) */
    const double x_bl = old_xs[0], p_bl = old_ps[0], x_tl = old_xs[2], p_tl = old_ps[2];
    const double x_br = old_xs[6], p_br = old_ps[6], x_tr = old_xs[8], p_tr = old_ps[8];
    double xt = x;
    int cnt = 0;
    while (!((x_tl - x_bl) * (p - p_bl) <= (p_tl - p_bl) * (xt - x_bl))) {
        xt += Lx;
        if (++cnt > 10) { *rc = -1; return 0.0; }
    }
    cnt = 0;
    while (!((x_tr - x_br) * (p - p_br) > (p_tr - p_br) * (xt - (x_br)))) {
        xt -= Lx;
        if (++cnt > 10) { *rc = -1; return 0.0; }
    }
    locate_ctx c = {old_m, old_xs, old_ps, Lx};
    int beyond = 0;
    const int l = find_recursive(&c, &xt, p, &beyond, 0);
    if (beyond || l == 0) return f_beyond;
    const opanel* P = &old_m->p[l];
    double px[9], pp[9], pf[9], k[9];
    for (int i = 0; i < 9; ++i) { px[i] = old_xs[P->pts[i]]; pp[i] = old_ps[P->pts[i]]; pf[i] = old_fs[P->pts[i]]; }
    fit_coefs(px, pp, pf, k);
    const double dx = xt - px[4], dp = p - pp[4];
    /* interpolate_from_panel's single-point expression (:1086-1088) */
    return k[0] + k[1] * dx + k[2] * dx * dp + k[3] * dp + k[4] * dx * dx + k[5] * dx * dx * dp +
           k[6] * dx * dx * dp * dp + k[7] * dx * dp * dp + k[8] * dp * dp;
}

/* test_panel (AMRStructure_amr.cpp:971-1081).  The p-derivative criterion of
 * the reference reads six entries of which it sets two (:1051-1061, the rest
 * are uninitialised); the restatement uses the two it sets. */
static void amr_test(fso_mesh* m, int pi, const double* f, const double* eps, int neps, int max_height) {
    opanel* P = &m->p[pi];
    double pf[9];
    for (int i = 0; i < 9; ++i) pf[i] = f[P->pts[i]];
    int crit = 0;
    if (neps > 0) {
        double mx = pf[0], mn = pf[0];
        for (int i = 1; i < 9; ++i) { if (mx < pf[i]) mx = pf[i]; if (mn > pf[i]) mn = pf[i]; }
        crit = crit || (mx - mn > eps[0]);
        if (neps > 1) crit = crit || (mx - mn) / pf[4] > eps[1];
        if (neps > 2) crit = crit || mx / mn > eps[2];
    }
    if (neps > 3) {
        const double dx = m->xs[P->pts[3]] - m->xs[P->pts[0]];
        double md = fabs((pf[3] - pf[0]) / dx);
        for (int i = 1; i < 6; ++i) { double v = fabs((pf[3 + i] - pf[i]) / dx); if (md < v) md = v; }
        crit = crit || (md > eps[3]);
    }
    if (neps > 4) {
        const double dp = m->ps[P->pts[1]] - m->ps[P->pts[0]];
        double a[2] = {0.0, 0.0};
        for (int jj = 0; jj < 3; ++jj)
            for (int ii = 0; ii < 2; ++ii) a[ii] = fabs((pf[3 * jj + ii + 1] - pf[3 * jj + ii]) / dp);
        const double md = a[0] < a[1] ? a[1] : a[0];
        crit = crit || (md > eps[4]);
    }
    if (P->level < max_height && crit) { P->needs = 1; m->need_further = 1; }
}

double* fso_mesh_adapt(fso_mesh* m, double* f, const double* eps, int neps, int max_height, fso_eval_fn eval,
                       void* ctx) {
    m->need_further = 0;
    for (int i = m->min_unrefined; i < m->np; ++i) amr_test(m, i, f, eps, neps, max_height);
    while (m->need_further) {
        m->need_further = 0;
        const int n0 = m->npts;
        mesh_refine_xp(m);
        f = (double*)realloc(f, sizeof(double) * (m->npts > 0 ? m->npts : 1));
        if (m->npts > n0) eval(ctx, m->xs + n0, m->ps + n0, m->npts - n0, f + n0);
        for (int i = m->min_unrefined; i < m->np; ++i)
            if (!m->p[i].xp) amr_test(m, i, f, eps, neps, max_height);
    }
    free(m->leaves);
    m->leaves = (int*)malloc(sizeof(int) * m->np);
    m->nleaves = 0;
    mesh_collect_leaves(m, 0);
    return f;
}

/* ======================================================================= */
/* Open-boundary direct sum and drive fields                                */
/* ======================================================================= */
void fso_direct_sum_open(double eps, double* es, const double* targets, int nt, const double* sources,
                         const double* q_ws, int ns) {
    const double e2 = eps * eps;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nt; ++i) {
        const double x = targets[i];
        double acc = 0.0;
        for (int j = 0; j < ns; ++j) {
            const double z = x - sources[j];
            acc += q_ws[j] * 0.5 * z / sqrt(z * z + e2);
        }
        es[i] = acc - x;
    }
}

/* ExternalTanh switches on around t = 69 and off around t = 307 (widths 20),
 * normalised so that it starts from zero at t = 0 (FieldStructure.cpp:17-36). */
static double tanh_switch(double t) { return 0.5 * (tanh((t - 69.0) / 20.0) - tanh((t - 307.0) / 20.0)); }

double fso_external_amplitude(int type, double Am, double k, double t) {
    if (type == 1) {  /* ExternalSine (:48-64): ramp up to t=50, hold to 150, ramp down to 200 */
        if (t < 50.0) return Am * sin(t * M_PI / 100);
        if (t < 150.0) return Am;
        if (t < 200.0) return Am * cos((t - 150) * M_PI / 100);
        return 0.0;
    }
    if (type == 2) {  /* ExternalLogistic (:70-84): logistic on at t=10, off at t=110 */
        if (t < 60.0) return Am / (1.0 + exp(-40.0 * (t - 10.0)));
        return Am * (1.0 - 1.0 / (1.0 + exp(-40.0 * (t - 110.0))));
    }
    const double e0 = tanh_switch(0.0);
    return (tanh_switch(t) - e0) / (1 - e0) * Am * k;
}

void fso_external_field(int type, double Am, double k, double omega, double* es, const double* x, int n,
                        double t) {
    const double a = fso_external_amplitude(type, Am, k, t);
    const double omt = omega * t;
    for (int i = 0; i < n; ++i) es[i] += a * sin(k * x[i] - omt);
}

/* ======================================================================= */
/* Reduced grid                                                             */
/* ======================================================================= */
static const double* g_rx;
static int cmp_x(const void* a, const void* b) {
    double xa = g_rx[*(const int*)a], xb = g_rx[*(const int*)b];
    return (xa < xb) ? -1 : (xa > xb) ? 1 : 0;
}
int fso_reduce(const double* xs, const double* q_ws, int n, double* rxs, double* rws, int* inv) {
    int* idx = (int*)malloc(sizeof(int) * n);
    for (int i = 0; i < n; ++i) idx[i] = i;
    g_rx = xs;
    qsort(idx, n, sizeof(int), cmp_x);
    double val = xs[idx[0]];
    int u = 0;
    rxs[0] = val;
    inv[idx[0]] = 0;
    for (int ii = 1; ii < n; ++ii) {
        int s = idx[ii];
        if (xs[s] > val) { val = xs[s]; u++; rxs[u] = val; }
        inv[s] = u;
    }
    const int nu = u + 1;
    for (int i = 0; i < nu; ++i) rws[i] = 0.0;
    for (int ii = 0; ii < n; ++ii) rws[inv[ii]] += q_ws[ii];
    free(idx);
    return nu;
}

/* ======================================================================= */
/* Simulation                                                               */
/* ======================================================================= */
struct fso_sim {
    fso_sim_params prm;
    fso_mesh* mesh[8];
    double* w0[8];
    double f_beyond[8];
    double qm[8];
    int start[9];
    int N;
    double *xs, *ps, *fs, *qws, *es;
    double Lx, t;
    int iter;
    long long full_evals, reduced_evals;
};

/* evaluate_field (AMRSimulation_field.cpp:164-173): the field, then the drive
 * field at time t on the same positions. */
static void sim_field(fso_sim* s, double* es, const double* x, const double* q, int n, double t) {
    const fso_sim_params* P = &s->prm;
    if (P->use_treecode) fso_treecode(s->Lx, P->greens_epsilon, P->mac, P->degree, P->max_source, es, x, q, n);
    else fso_direct_sum(s->Lx, P->greens_epsilon, es, x, n, x, q, n);
    if (P->use_external_field)
        fso_external_field(P->external_type, P->ext_Am, P->ext_k, P->ext_omega, es, x, n, t);
}

/* evaluate_field_uniform_grid (src/simulation_files/AMRSimulation_field.cpp:5-162). */
static void sim_reduced_field(fso_sim* s) {
    const int ns = s->prm.num_species;
    double* rx = (double*)malloc(sizeof(double) * s->N);
    double* rw = (double*)malloc(sizeof(double) * s->N);
    int* inv = (int*)malloc(sizeof(int) * s->N);
    int off[9];
    int tot = 0;
    for (int sp = 0; sp < ns; ++sp) {
        int a = s->start[sp], n = s->start[sp + 1] - a;
        off[sp] = tot;
        tot += fso_reduce(s->xs + a, s->qws + a, n, rx + tot, rw + tot, inv + a);
    }
    off[ns] = tot;
    double* re = (double*)malloc(sizeof(double) * tot);
    sim_field(s, re, rx, rw, tot, s->t);
    s->reduced_evals++;
    for (int sp = 0; sp < ns; ++sp)
        for (int i = s->start[sp]; i < s->start[sp + 1]; ++i) s->es[i] = re[off[sp] + inv[i]];
    free(rx); free(rw); free(inv); free(re);
}

typedef struct { const fso_dist* d; int rc; } f0_ctx;
static void eval_f0(void* ctx, const double* x, const double* p, int n, double* out) {
    f0_ctx* c = (f0_ctx*)ctx;
    for (int i = 0; i < n; ++i) {
        int rc = 0;
        out[i] = fso_dist_eval(c->d, x[i], p[i], &rc);
        if (rc) c->rc = rc;
    }
}
typedef struct {
    const fso_mesh* old_m;
    const double *ox, *op, *of;
    double f_beyond;
    int rc;
} interp_ctx;
static void eval_interp(void* ctx, const double* x, const double* p, int n, double* out) {
    interp_ctx* c = (interp_ctx*)ctx;
    for (int i = 0; i < n; ++i) {
        int rc = 0;
        out[i] = fso_interp_point(c->old_m, c->ox, c->op, c->of, c->f_beyond, x[i], p[i], &rc);
        if (rc) c->rc = rc;
    }
}

fso_sim* fso_sim_create(const fso_sim_params* prm) {
    if (prm->num_species < 1 || prm->num_species > 8) return NULL;
    fso_sim* s = (fso_sim*)calloc(1, sizeof(fso_sim));
    s->prm = *prm;
    s->Lx = prm->xmax - prm->xmin;
    int tot = 0;
    double* f_init[8] = {0};
    for (int sp = 0; sp < prm->num_species; ++sp) {
        const fso_species_params* q = &prm->species[sp];
        s->mesh[sp] = fso_mesh_build(q->initial_height, q->p_height, prm->xmin, prm->xmax, q->pmin, q->pmax);
        if (!s->mesh[sp]) { fso_sim_destroy(s); return NULL; }
        /* the initial condition (AMRStructure ctor / generate_mesh at the initial step) */
        int drc = 0;
        fso_dist* dist = fso_dist_create(q, prm->xmin, prm->xmax, &drc);
        if (!dist) { fso_sim_destroy(s); return NULL; }
        fso_mesh* m = s->mesh[sp];
        f0_ctx fc = {dist, 0};
        double* f = (double*)malloc(sizeof(double) * m->npts);
        eval_f0(&fc, m->xs, m->ps, m->npts, f);
        /* fso_mesh_adapt reallocates f and returns it */
        f_init[sp] = (q->do_adaptively_refine && q->n_amr_eps > 0)
                         ? fso_mesh_adapt(m, f, q->amr_eps, q->n_amr_eps, q->max_height, eval_f0, &fc)
                         : f;
        fso_dist_destroy(dist);
        if (fc.rc) { for (int k = 0; k <= sp; ++k) free(f_init[k]); fso_sim_destroy(s); return NULL; }
        s->start[sp] = tot;
        tot += s->mesh[sp]->npts;
    }
    s->start[prm->num_species] = tot;
    s->N = tot;
    s->xs = (double*)malloc(sizeof(double) * tot);
    s->ps = (double*)malloc(sizeof(double) * tot);
    s->fs = (double*)malloc(sizeof(double) * tot);
    s->qws = (double*)malloc(sizeof(double) * tot);
    s->es = (double*)calloc(tot, sizeof(double));
    for (int sp = 0; sp < prm->num_species; ++sp) {
        const fso_species_params* q = &prm->species[sp];
        const fso_mesh* m = s->mesh[sp];
        const int a = s->start[sp];
        s->qm[sp] = q->q / q->m;
        s->w0[sp] = (double*)malloc(sizeof(double) * m->npts);
        fso_mesh_base_weights(m, q->q, prm->quadrature, s->w0[sp]);
        double fmin = 0;
        for (int i = 0; i < m->npts; ++i) {
            s->xs[a + i] = m->xs[i];
            s->ps[a + i] = m->ps[i];
            s->fs[a + i] = f_init[sp][i];
            s->qws[a + i] = s->w0[sp][i] * s->fs[a + i];
            if (i == 0 || s->fs[a + i] < fmin) fmin = s->fs[a + i];
        }
        free(f_init[sp]);
        s->f_beyond[sp] = fmin;  /* AMRStructure.cpp:124 */
    }
    sim_reduced_field(s);
    return s;
}

void fso_sim_destroy(fso_sim* s) {
    if (!s) return;
    for (int sp = 0; sp < 8; ++sp) { fso_mesh_destroy(s->mesh[sp]); free(s->w0[sp]); }
    free(s->xs); free(s->ps); free(s->fs); free(s->qws); free(s->es);
    free(s);
}

/* relativistic_momentum_push's velocity (AMRSimulation_step.cpp:101-111):
 * v = (p/m) / sqrt(1 + (p/m)^2) with the species mass m */
static void push_velocity(const fso_sim* s, const double* p, double* v) {
    for (int sp = 0; sp < s->prm.num_species; ++sp) {
        const double m = s->prm.species[sp].m;
        for (int i = s->start[sp]; i < s->start[sp + 1]; ++i) {
            const double u = p[i] / m;
            v[i] = u / sqrt(1 + u * u);
        }
    }
}

/* AMRSimulation::rk4_step (src/simulation_files/AMRSimulation_step.cpp:122-263). */
static void sim_rk4(fso_sim* s) {
    const int N = s->N, ns = s->prm.num_species;
    const double dt = s->prm.dt;
    double* xk = (double*)malloc(sizeof(double) * N);
    double* p1 = (double*)malloc(sizeof(double) * N);
    double* p2 = (double*)malloc(sizeof(double) * N);
    double* p3 = (double*)malloc(sizeof(double) * N);
    double* p4 = (double*)malloc(sizeof(double) * N);
    double* e1 = (double*)malloc(sizeof(double) * N);
    double* e2 = (double*)malloc(sizeof(double) * N);
    double* e3 = (double*)malloc(sizeof(double) * N);
    double* e4 = (double*)malloc(sizeof(double) * N);
    memcpy(p1, s->ps, sizeof(double) * N);
    memcpy(e1, s->es, sizeof(double) * N);
    /* v1..v4: the stage momenta, or with the relativistic push their velocities */
    double* v1 = p1; double* v2 = p2; double* v3 = p3; double* v4 = p4;
    const int rel = s->prm.relativistic_push != 0;
    if (rel) {
        v1 = (double*)malloc(sizeof(double) * N);
        v2 = (double*)malloc(sizeof(double) * N);
        v3 = (double*)malloc(sizeof(double) * N);
        v4 = (double*)malloc(sizeof(double) * N);
        push_velocity(s, p1, v1);
    }
    for (int sp = 0; sp < ns; ++sp)
        for (int i = s->start[sp]; i < s->start[sp + 1]; ++i) {
            e1[i] *= s->qm[sp];
            p2[i] = s->ps[i] + 0.5 * dt * e1[i];
            xk[i] = s->xs[i] + 0.5 * dt * v1[i];
        }
    if (rel) push_velocity(s, p2, v2);
    const double t2 = s->t + dt * 0.5, t4 = s->t + dt;  /* rk4_step :170, :201, :224 */
    sim_field(s, e2, xk, s->qws, N, t2);
    for (int sp = 0; sp < ns; ++sp)
        for (int i = s->start[sp]; i < s->start[sp + 1]; ++i) {
            e2[i] *= s->qm[sp];
            p3[i] = s->ps[i] + 0.5 * dt * e2[i];
            xk[i] = s->xs[i] + 0.5 * dt * v2[i];
        }
    if (rel) push_velocity(s, p3, v3);
    sim_field(s, e3, xk, s->qws, N, t2);
    for (int sp = 0; sp < ns; ++sp)
        for (int i = s->start[sp]; i < s->start[sp + 1]; ++i) {
            e3[i] *= s->qm[sp];
            p4[i] = s->ps[i] + dt * e3[i];
            xk[i] = s->xs[i] + dt * v3[i];
        }
    if (rel) push_velocity(s, p4, v4);
    sim_field(s, e4, xk, s->qws, N, t4);
    s->full_evals += 3;
    for (int sp = 0; sp < ns; ++sp)
        for (int i = s->start[sp]; i < s->start[sp + 1]; ++i) e4[i] *= s->qm[sp];
    for (int i = 0; i < N; ++i) {
        s->xs[i] += dt / 6.0 * (v1[i] + 2 * v2[i] + 2 * v3[i] + v4[i]);
        s->ps[i] += dt / 6.0 * (e1[i] + 2 * e2[i] + 2 * e3[i] + e4[i]);
    }
    if (rel) { free(v1); free(v2); free(v3); free(v4); }
    free(xk); free(p1); free(p2); free(p3); free(p4); free(e1); free(e2); free(e3); free(e4);
}

/* AMRSimulation::remesh (src/simulation_files/AMRSimulation_remesh.cpp:3-48)
 * with AMRStructure::remesh (AMRStructure_amr.cpp:1156-1202). */
static int sim_remesh(fso_sim* s) {
    const int ns = s->prm.num_species;
    double *nx[8], *np_[8], *nf[8], *nq[8];
    int cnt[8];
    int rc = 0;
    for (int sp = 0; sp < ns; ++sp) {
        const fso_species_params* q = &s->prm.species[sp];
        fso_mesh* m = s->mesh[sp];
        const int a = s->start[sp];
        if (q->do_adaptively_refine && q->n_amr_eps > 0) {
            /* generate_mesh after a step: the uniform base mesh, f interpolated
             * at its lattice, then adaptive refinement with interpolate_from_mesh */
            fso_mesh* nm = fso_mesh_build(q->initial_height, q->p_height, s->prm.xmin, s->prm.xmax, q->pmin, q->pmax);
            double* f = (double*)malloc(sizeof(double) * nm->npts);
            rc = fso_remesh_interp2(m, nm, s->xs + a, s->ps + a, s->fs + a, s->f_beyond[sp], f);
            if (rc) { free(f); fso_mesh_destroy(nm); break; }
            interp_ctx ic = {m, s->xs + a, s->ps + a, s->fs + a, s->f_beyond[sp], 0};
            f = fso_mesh_adapt(nm, f, q->amr_eps, q->n_amr_eps, q->max_height, eval_interp, &ic);
            if (ic.rc) { free(f); fso_mesh_destroy(nm); rc = ic.rc; break; }
            free(s->w0[sp]);
            s->w0[sp] = (double*)malloc(sizeof(double) * nm->npts);
            fso_mesh_base_weights(nm, q->q, s->prm.quadrature, s->w0[sp]);
            fso_mesh_destroy(m);
            s->mesh[sp] = nm;
            m = nm;
            nf[sp] = f;
        } else {
            nf[sp] = (double*)malloc(sizeof(double) * m->npts);
            rc = fso_remesh_interp(m, s->xs + a, s->ps + a, s->fs + a, s->f_beyond[sp], nf[sp], NULL, NULL);
            if (rc) { free(nf[sp]); break; }
        }
        cnt[sp] = m->npts;
        nx[sp] = (double*)malloc(sizeof(double) * cnt[sp]);
        np_[sp] = (double*)malloc(sizeof(double) * cnt[sp]);
        nq[sp] = (double*)malloc(sizeof(double) * cnt[sp]);
        for (int i = 0; i < cnt[sp]; ++i) {
            nx[sp][i] = m->xs[i];
            np_[sp][i] = m->ps[i];
            nq[sp][i] = s->w0[sp][i] * nf[sp][i];
        }
    }
    if (rc) return rc;  /* (the partial buffers are released with the failed run) */
    /* relayout: species concatenated in deck order */
    int tot = 0;
    for (int sp = 0; sp < ns; ++sp) { s->start[sp] = tot; tot += cnt[sp]; }
    s->start[ns] = tot;
    s->N = tot;
    free(s->xs); free(s->ps); free(s->fs); free(s->qws); free(s->es);
    s->xs = (double*)malloc(sizeof(double) * tot);
    s->ps = (double*)malloc(sizeof(double) * tot);
    s->fs = (double*)malloc(sizeof(double) * tot);
    s->qws = (double*)malloc(sizeof(double) * tot);
    s->es = (double*)calloc(tot, sizeof(double));
    for (int sp = 0; sp < ns; ++sp) {
        const int a = s->start[sp];
        memcpy(s->xs + a, nx[sp], sizeof(double) * cnt[sp]);
        memcpy(s->ps + a, np_[sp], sizeof(double) * cnt[sp]);
        memcpy(s->fs + a, nf[sp], sizeof(double) * cnt[sp]);
        memcpy(s->qws + a, nq[sp], sizeof(double) * cnt[sp]);
        free(nx[sp]); free(np_[sp]); free(nf[sp]); free(nq[sp]);
    }
    sim_reduced_field(s);
    return 0;
}

int fso_sim_step(fso_sim* s) {
    sim_rk4(s);
    s->iter += 1;
    s->t += s->prm.dt;
    if (s->iter % s->prm.remesh_period == 0) return sim_remesh(s);
    sim_field(s, s->es, s->xs, s->qws, s->N, s->t);
    s->full_evals += 1;
    return 0;
}

int fso_sim_total_points(const fso_sim* s) { return s->N; }
int fso_sim_species_points(const fso_sim* s, int sp) { return s->start[sp + 1] - s->start[sp]; }
int fso_sim_iter(const fso_sim* s) { return s->iter; }
void fso_sim_state(const fso_sim* s, double* xs, double* ps, double* fs, double* q_ws, double* es) {
    size_t b = sizeof(double) * s->N;
    if (xs) memcpy(xs, s->xs, b);
    if (ps) memcpy(ps, s->ps, b);
    if (fs) memcpy(fs, s->fs, b);
    if (q_ws) memcpy(q_ws, s->qws, b);
    if (es) memcpy(es, s->es, b);
}
void fso_sim_counters(const fso_sim* s, long long* full, long long* reduced) {
    if (full) *full = s->full_evals;
    if (reduced) *reduced = s->reduced_evals;
}
