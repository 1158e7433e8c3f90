/*
 * exact_tritri.c -- exact triangle-triangle intersection decision for FP32
 * input, used as the "FP64 exact-predicate" oracle.
 *
 * TEST INFRASTRUCTURE ONLY (see bvhcd_oracle.h).
 *
 * Method: the 17 candidate separating axes of the triangle SAT (two face
 * normals, nine edge-edge cross products, six in-plane edge normals), each
 * evaluated exactly.  Every projection difference a.(P_i - Q_j) is a
 * polynomial in the input coordinates; it is computed without rounding as a
 * floating-point expansion (a sum of non-overlapping doubles) with the
 * error-free transformations Two-Sum and Two-Product and the expansion sum /
 * scale algorithms published by J. R. Shewchuk, "Adaptive Precision
 * Floating-Point Arithmetic and Fast Robust Geometric Predicates" (1997).
 * The sign of an expansion is the sign of its largest component.
 * Two closed triangles are disjoint iff some axis strictly separates their
 * projections; a zero axis never separates.  Compile without
 * -ffast-math and with -ffp-contract=off.
 */
#include <math.h>
#include <string.h>

#include "bvhcd_oracle.h"

#define EXP_MAX 4096

typedef struct { int n; double c[EXP_MAX]; } expn; /* increasing magnitude */

static inline void two_sum(double a, double b, double *s, double *e) {
    double x = a + b, bv = x - a, av = x - bv;
    *s = x;
    *e = (a - av) + (b - bv);
}
static inline void fast_two_sum(double a, double b, double *s, double *e) {
    double x = a + b;
    *s = x;
    *e = b - (x - a);
}
static inline void two_prod(double a, double b, double *p, double *e) {
    double x = a * b;
    *p = x;
    *e = fma(a, b, -x);
}

/* Grow-Expansion applied for each component of f (Expansion-Sum), with zero
 * elimination.  h may not alias e or f. */
static void exp_add(const expn *e, const expn *f, expn *h) {
    double tmp[2 * EXP_MAX];
    int n = e->n;
    memcpy(tmp, e->c, sizeof(double) * (size_t)n);
    for (int j = 0; j < f->n; j++) {
        double q = f->c[j];
        int m = 0;
        for (int i = 0; i < n; i++) {
            double s, err;
            two_sum(q, tmp[i], &s, &err);
            q = s;
            if (err != 0.0) tmp[m++] = err;
        }
        if (q != 0.0 || m == 0) tmp[m++] = q;
        n = m;
    }
    if (n == 1 && tmp[0] == 0.0) n = 0;
    if (n > EXP_MAX) n = EXP_MAX; /* not reached for degree <= 4 inputs */
    h->n = n;
    memcpy(h->c, tmp, sizeof(double) * (size_t)n);
}

/* Scale-Expansion with zero elimination */
static void exp_scale(const expn *e, double b, expn *h) {
    int m = 0;
    if (e->n == 0 || b == 0.0) { h->n = 0; return; }
    double Q, hh;
    two_prod(e->c[0], b, &Q, &hh);
    if (hh != 0.0) h->c[m++] = hh;
    for (int i = 1; i < e->n; i++) {
        double T, t, s;
        two_prod(e->c[i], b, &T, &t);
        two_sum(Q, t, &s, &hh);
        if (hh != 0.0) h->c[m++] = hh;
        fast_two_sum(T, s, &Q, &hh);
        if (hh != 0.0) h->c[m++] = hh;
    }
    if (Q != 0.0 || m == 0) h->c[m++] = Q;
    if (m == 1 && h->c[0] == 0.0) m = 0;
    h->n = m;
}

static inline void exp_copy(expn *dst, const expn *src) {
    dst->n = src->n;
    memcpy(dst->c, src->c, sizeof(double) * (size_t)src->n);
}

static void exp_mul(const expn *e, const expn *f, expn *h) {
    static __thread expn acc, part, tmp;
    acc.n = 0;
    for (int j = 0; j < f->n; j++) {
        exp_scale(e, f->c[j], &part);
        exp_add(&acc, &part, &tmp);
        exp_copy(&acc, &tmp);
    }
    exp_copy(h, &acc);
}
static void exp_neg(expn *e) {
    for (int i = 0; i < e->n; i++) e->c[i] = -e->c[i];
}
static void exp_sub(const expn *e, const expn *f, expn *h) {
    static __thread expn nf;
    exp_copy(&nf, f);
    exp_neg(&nf);
    exp_add(e, &nf, h);
}
static int exp_sign(const expn *e) {
    for (int i = e->n - 1; i >= 0; i--) {
        if (e->c[i] > 0) return 1;
        if (e->c[i] < 0) return -1;
    }
    return 0;
}
static void exp_diff(double a, double b, expn *h) { /* exact a - b */
    double s, e;
    two_sum(a, -b, &s, &e);
    h->n = 0;
    if (e != 0.0) h->c[h->n++] = e;
    if (s != 0.0) h->c[h->n++] = s;
}

typedef struct { expn v[3]; } evec;

static void ev_cross(const evec *a, const evec *b, evec *r) {
    static __thread expn t1, t2;
    exp_mul(&a->v[1], &b->v[2], &t1); exp_mul(&a->v[2], &b->v[1], &t2); exp_sub(&t1, &t2, &r->v[0]);
    exp_mul(&a->v[2], &b->v[0], &t1); exp_mul(&a->v[0], &b->v[2], &t2); exp_sub(&t1, &t2, &r->v[1]);
    exp_mul(&a->v[0], &b->v[1], &t1); exp_mul(&a->v[1], &b->v[0], &t2); exp_sub(&t1, &t2, &r->v[2]);
}
static void ev_dot(const evec *a, const evec *b, expn *r) {
    static __thread expn t, s1, s2;
    exp_mul(&a->v[0], &b->v[0], &s1);
    exp_mul(&a->v[1], &b->v[1], &t);
    exp_add(&s1, &t, &s2);
    exp_mul(&a->v[2], &b->v[2], &t);
    exp_add(&s2, &t, r);
}

/* 1 when the axis separates (all a.(P_i-Q_j) > 0, or all < 0) */
static int separates(const evec *ax, const evec d[3][3]) {
    static __thread expn pr;
    int pos = 0, neg = 0;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            ev_dot(ax, &d[i][j], &pr);
            int s = exp_sign(&pr);
            if (s > 0) pos++;
            else if (s < 0) neg++;
            else return 0;
            if (pos && neg) return 0;
        }
    return 1;
}

int orc_tritri_exact(const float *P, const float *Q) {
    static __thread evec e[3], f[3], n, m, ax, d[3][3];
    for (int k = 0; k < 3; k++) {
        int k1 = (k + 1) % 3;
        for (int c = 0; c < 3; c++) {
            exp_diff((double)P[3 * k1 + c], (double)P[3 * k + c], &e[k].v[c]);
            exp_diff((double)Q[3 * k1 + c], (double)Q[3 * k + c], &f[k].v[c]);
        }
    }
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++)
            for (int c = 0; c < 3; c++)
                exp_diff((double)P[3 * i + c], (double)Q[3 * j + c], &d[i][j].v[c]);
    ev_cross(&e[0], &e[1], &n);
    ev_cross(&f[0], &f[1], &m);
    if (separates(&n, d)) return 0;
    if (separates(&m, d)) return 0;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            ev_cross(&e[i], &f[j], &ax);
            if (separates(&ax, d)) return 0;
        }
    for (int i = 0; i < 3; i++) {
        ev_cross(&e[i], &n, &ax);
        if (separates(&ax, d)) return 0;
    }
    for (int j = 0; j < 3; j++) {
        ev_cross(&f[j], &m, &ax);
        if (separates(&ax, d)) return 0;
    }
    return 1;
}
