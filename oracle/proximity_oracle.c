/*
 * proximity_oracle.c -- CPU reference of bvhcd_front_proximity (test
 * infrastructure only: the checker of the CUDA proximity kernel).
 *
 * signed_vf_distance and signed_ee_distance (Mine/utility/CudaDeviceUtils.cu:
 * 163-193, proj = v . (p0 x p1), Mine/utility/CudaDeviceUtils.h:66-68),
 * restated in double with one rounding per operation (built with
 * -ffp-contract=off; sqrt and division are correctly rounded), the operations
 * in the order of the CUDA kernel, so the two agree bit for bit.  For a
 * triangle pair, the 15 feature pairs in the kernel's order: each vertex of
 * the first against the second's face, each vertex of the second against the
 * first's face, each edge of the first against each edge of the second.  A
 * feature pair is kept when its signed distance is within the thickness and
 * every barycentric weight is non-negative; feature pairs of one mesh that
 * share a vertex id are skipped.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>

#include "bvhcd_oracle.h"

typedef struct { double x, y, z; } p3;

static inline p3 psub(p3 a, p3 b) { p3 r = {a.x - b.x, a.y - b.y, a.z - b.z}; return r; }
static inline p3 pscale(p3 a, double s) { p3 r = {a.x * s, a.y * s, a.z * s}; return r; }
static inline double pdot(p3 a, p3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline p3 pcross(p3 a, p3 b) {
    p3 r = {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
    return r;
}
static inline p3 pnormalize(p3 v) { return pscale(v, 1.0 / sqrt(pdot(v, v))); }
static inline double pproj(p3 v, p3 p0, p3 p1) { return pdot(v, pcross(p0, p1)); }

static int vf(p3 x, p3 y0, p3 y1, p3 y2, double *d, p3 *n, double w[4]) {
    *n = pcross(pnormalize(psub(y1, y0)), pnormalize(psub(y2, y0)));
    if (!(pdot(*n, *n) >= DBL_EPSILON)) return 0;
    *n = pnormalize(*n);
    double b0 = pproj(psub(y1, x), psub(y2, x), *n);
    double b1 = pproj(psub(y2, x), psub(y0, x), *n);
    double b2 = pproj(psub(y0, x), psub(y1, x), *n);
    double s = (b0 + b1) + b2;
    w[0] = 1.0;
    w[1] = -(b0 / s);
    w[2] = -(b1 / s);
    w[3] = -(b2 / s);
    *d = pdot(psub(x, y0), *n);
    return 1;
}

static int ee(p3 x0, p3 x1, p3 y0, p3 y1, double *d, p3 *n, double w[4]) {
    *n = pcross(pnormalize(psub(x1, x0)), pnormalize(psub(y1, y0)));
    if (!(pdot(*n, *n) >= (double)FLT_EPSILON)) return 0;
    *n = pnormalize(*n);
    double a0 = pproj(psub(y1, x1), psub(y0, x1), *n);
    double a1 = pproj(psub(y0, x0), psub(y1, x0), *n);
    double b0 = pproj(psub(x0, y1), psub(x1, y1), *n);
    double b1 = pproj(psub(x1, y0), psub(x0, y0), *n);
    double sa = a0 + a1, sb = b0 + b1;
    w[0] = a0 / sa;
    w[1] = a1 / sa;
    w[2] = -(b0 / sb);
    w[3] = -(b1 / sb);
    *d = pdot(psub(x0, y0), *n);
    return 1;
}

static void put(orc_prox *out, int64_t cap, int64_t *k, int pair, int kind, int fa, int fb, double d, p3 n,
                const double w[4]) {
    if (*k < cap && out) {
        orc_prox *r = out + *k;
        r->pair = pair; r->kind = kind; r->fa = fa; r->fb = fb;
        r->dist = d;
        r->n[0] = n.x; r->n[1] = n.y; r->n[2] = n.z;
        for (int i = 0; i < 4; i++) r->w[i] = w[i];
    }
    (*k)++;
}

int64_t orc_proximity(int64_t n, const int *pairs, const int *fa, const float *va, const int *fb, const float *vb,
                      int same_mesh, double h, orc_prox *out, int64_t cap) {
    int64_t k = 0;
    for (int64_t q = 0; q < n; q++) {
        const int ta = pairs[2 * q], tb = pairs[2 * q + 1];
        int ia[3], ib[3];
        p3 pa[3], pb[3];
        for (int v = 0; v < 3; v++) {
            ia[v] = fa[3 * (int64_t)ta + v];
            ib[v] = fb[3 * (int64_t)tb + v];
            const float *x = va + 3 * (int64_t)ia[v], *y = vb + 3 * (int64_t)ib[v];
            p3 xa = {x[0], x[1], x[2]}, yb = {y[0], y[1], y[2]};
            pa[v] = xa;
            pb[v] = yb;
        }
        double d, w[4];
        p3 nn;
        for (int i = 0; i < 3; i++) {
            if (same_mesh && (ia[i] == ib[0] || ia[i] == ib[1] || ia[i] == ib[2])) continue;
            if (vf(pa[i], pb[0], pb[1], pb[2], &d, &nn, w) && fabs(d) <= h && -w[1] >= 0.0 && -w[2] >= 0.0 &&
                -w[3] >= 0.0)
                put(out, cap, &k, (int)q, 0, i, -1, d, nn, w);
        }
        for (int j = 0; j < 3; j++) {
            if (same_mesh && (ib[j] == ia[0] || ib[j] == ia[1] || ib[j] == ia[2])) continue;
            if (vf(pb[j], pa[0], pa[1], pa[2], &d, &nn, w) && fabs(d) <= h && -w[1] >= 0.0 && -w[2] >= 0.0 &&
                -w[3] >= 0.0)
                put(out, cap, &k, (int)q, 1, -1, j, d, nn, w);
        }
        for (int i = 0; i < 3; i++) {
            const int i1 = i == 2 ? 0 : i + 1;
            for (int j = 0; j < 3; j++) {
                const int j1 = j == 2 ? 0 : j + 1;
                if (same_mesh && (ia[i] == ib[j] || ia[i] == ib[j1] || ia[i1] == ib[j] || ia[i1] == ib[j1]))
                    continue;
                if (ee(pa[i], pa[i1], pb[j], pb[j1], &d, &nn, w) && fabs(d) <= h && w[0] >= 0.0 && w[1] >= 0.0 &&
                    -w[2] >= 0.0 && -w[3] >= 0.0)
                    put(out, cap, &k, (int)q, 2, i, j, d, nn, w);
            }
        }
    }
    return k;
}
