/*
 * sdot_oracle.c -- CPU restatement of the reference's 2D power-diagram path.
 *
 * TEST INFRASTRUCTURE ONLY (the parity reference; see sdot_oracle.h).  Pinned by
 * tests/test_oracle_kat.py against the known answers of the reference's own
 * tests (tests/test_ConvexPolyhedron2.cpp, tests/test_scaled_image.cpp) and,
 * where the reference compiles, against its outputs on seeded inputs.
 *
 * Restated reference functions (paths relative to the reference root):
 *   ConvexPolyhedron2( Box )              src/sdot/Geometry/ConvexPolyhedron2.tcc:76-106
 *   ConvexPolyhedron2( Simplex )          ConvexPolyhedron2.tcc:19-60
 *   plane_cut                             ConvexPolyhedron2.tcc:687-924
 *   ball_cut                              ConvexPolyhedron2.tcc:534-666
 *   intersect_with                        ConvexPolyhedron2.tcc:2475-2496
 *   integration( Constant, Unit )         ConvexPolyhedron2.tcc:1791-1843
 *   integration( Polynomial<6>, Unit )    ConvexPolyhedron2.tcc:2181-2225 (as triangle moments)
 *   add_centroid_contrib( Constant,Unit ) ConvexPolyhedron2.tcc:1047-1074
 *   for_each_boundary_item( Constant,Unit) ConvexPolyhedron2.tcc:437-478
 *   _arc_area / _centroid_arc / _arc_length ConvexPolyhedron2.tcc:2296-2381
 *   min_position / max_position           ConvexPolyhedron2.tcc:502-524
 *   weighted bisector cut                 src/sdot/PowerDiagram/Visitors/SpZGrid.tcc:506-522
 *   eviction test                         SpZGrid.tcc:475-480
 *   get_integrals / get_centroids         src/sdot/PowerDiagram/get_integrals.h:12-21, get_centroids.h:46-55
 *   get_der_integrals_wrt_weights         src/sdot/PowerDiagram/get_der_integrals_wrt_weights.h:36-119
 *   ConvexPolyhedronAssembly              src/sdot/Domains/ConvexPolyhedronAssembly.tcc:7-142
 *   ScaledImage::for_each_intersection    src/sdot/Domains/ScaledImage.tcc:98-149 (full-disc bbox fixed)
 *
 * The neighbour search differs from SpZGrid's tree: a uniform grid is
 * scanned ring by ring, each grid cell skipped by the reference's eviction
 * test, and the scan stops when no Dirac beyond the current ring can reach
 * the cell (bound with the global maximum weight).  The resulting cell is the
 * same convex set; only the order of the cuts differs.
 */
#include "sdot_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

enum { LINE = 0, ARC = 1 };

struct or_poly {
    int n, cap;
    double *x, *y, *nx, *ny;
    int64_t *id;
    unsigned char *arc;
    double scx, scy, sr;
    int64_t sid;
    double *dist; /* work */
    unsigned char *out;
};

static void poly_reserve(or_poly *p, int cap) {
    if (cap <= p->cap) return;
    int c = cap < 64 ? 64 : 2 * cap;
    p->x = realloc(p->x, c * sizeof(double));
    p->y = realloc(p->y, c * sizeof(double));
    p->nx = realloc(p->nx, c * sizeof(double));
    p->ny = realloc(p->ny, c * sizeof(double));
    p->id = realloc(p->id, c * sizeof(int64_t));
    p->arc = realloc(p->arc, c);
    p->dist = realloc(p->dist, c * sizeof(double));
    p->out = realloc(p->out, c);
    for (int k = p->cap; k < c; ++k) p->arc[k] = 0;
    p->cap = c;
}

static or_poly *poly_new(void) {
    or_poly *p = calloc(1, sizeof(or_poly));
    poly_reserve(p, 64);
    return p;
}

static void poly_box_into(or_poly *p, double x0, double y0, double x1, double y1, int64_t cut_id) {
    poly_reserve(p, 4);
    p->scx = 0.5 * (x0 + x1);
    p->scy = 0.5 * (y0 + y1);
    p->sr = -1;
    p->sid = -1;
    p->n = 4;
    double xs[4] = {x0, x1, x1, x0}, ys[4] = {y0, y0, y1, y1};
    double nxs[4] = {0, 1, 0, -1}, nys[4] = {-1, 0, 1, 0};
    for (int k = 0; k < 4; ++k) {
        p->x[k] = xs[k]; p->y[k] = ys[k];
        p->nx[k] = nxs[k]; p->ny[k] = nys[k];
        p->id[k] = cut_id;
    }
    /* a freshly constructed polygon has no arc flag anywhere */
    memset(p->arc, 0, p->cap);
}

or_poly *or_poly_box(double x0, double y0, double x1, double y1, int64_t cut_id) {
    or_poly *p = poly_new();
    poly_box_into(p, x0, y0, x1, y1, cut_id);
    return p;
}

or_poly *or_poly_simplex(const double *q, int64_t cut_id) {
    or_poly *p = poly_new();
    p->scx = 1.0 / 3 * (q[0] + q[2] + q[4]);
    p->scy = 1.0 / 3 * (q[1] + q[3] + q[5]);
    p->sr = -1;
    p->sid = -1;
    p->n = 3;
    double n0[2], n1[2], n2[2];
    const double *a = q, *b = q + 2, *c = q + 4;
    /* rot90( p ) = ( -p.y, p.x ), then normalised */
    double v[2];
    v[0] = a[0] - b[0]; v[1] = a[1] - b[1]; n0[0] = -v[1]; n0[1] = v[0];
    v[0] = b[0] - c[0]; v[1] = b[1] - c[1]; n1[0] = -v[1]; n1[1] = v[0];
    v[0] = c[0] - a[0]; v[1] = c[1] - a[1]; n2[0] = -v[1]; n2[1] = v[0];
    double l;
    l = sqrt(n0[0] * n0[0] + n0[1] * n0[1]); n0[0] /= l; n0[1] /= l;
    l = sqrt(n1[0] * n1[0] + n1[1] * n1[1]); n1[0] /= l; n1[1] /= l;
    l = sqrt(n2[0] * n2[0] + n2[1] * n2[1]); n2[0] /= l; n2[1] /= l;
    p->x[0] = a[0]; p->y[0] = a[1];
    p->x[1] = b[0]; p->y[1] = b[1];
    p->x[2] = c[0]; p->y[2] = c[1];
    if ((a[0] - p->scx) * n0[0] + (a[1] - p->scy) * n0[1] < 0) {
        p->x[1] = c[0]; p->y[1] = c[1];
        p->x[2] = b[0]; p->y[2] = b[1];
        double t0 = n0[0], t1 = n0[1];
        n0[0] = -n2[0]; n0[1] = -n2[1];
        n1[0] = -n1[0]; n1[1] = -n1[1];
        n2[0] = -t0; n2[1] = -t1;
    }
    p->nx[0] = n0[0]; p->ny[0] = n0[1];
    p->nx[1] = n1[0]; p->ny[1] = n1[1];
    p->nx[2] = n2[0]; p->ny[2] = n2[1];
    for (int k = 0; k < 3; ++k) { p->id[k] = cut_id; p->arc[k] = 0; }
    return p;
}

static void poly_copy_into(or_poly *d, const or_poly *s) {
    poly_reserve(d, s->n);
    d->n = s->n;
    memcpy(d->x, s->x, s->n * sizeof(double));
    memcpy(d->y, s->y, s->n * sizeof(double));
    memcpy(d->nx, s->nx, s->n * sizeof(double));
    memcpy(d->ny, s->ny, s->n * sizeof(double));
    memcpy(d->id, s->id, s->n * sizeof(int64_t));
    memcpy(d->arc, s->arc, s->n);
    /* the reference copies the whole arc bitset (all zeros past the vertices
     * of a starting polygon): plane_cut never moves arc flags */
    memset(d->arc + s->n, 0, d->cap - s->n);
    d->scx = s->scx; d->scy = s->scy; d->sr = s->sr; d->sid = s->sid;
}

or_poly *or_poly_copy(const or_poly *s) {
    or_poly *p = poly_new();
    poly_copy_into(p, s);
    return p;
}

void or_poly_free(or_poly *p) {
    if (!p) return;
    free(p->x); free(p->y); free(p->nx); free(p->ny); free(p->id); free(p->arc); free(p->dist); free(p->out);
    free(p);
}

int or_poly_nb_points(const or_poly *p) { return p->n; }
double or_poly_sphere_radius(const or_poly *p) { return p->sr; }

void or_poly_points(const or_poly *p, double *xy, int64_t *ids, int *arcs) {
    for (int k = 0; k < p->n; ++k) {
        if (xy) { xy[2 * k] = p->x[k]; xy[2 * k + 1] = p->y[k]; }
        if (ids) ids[k] = p->id[k];
        if (arcs) arcs[k] = p->arc[k];
    }
}

static void mv(or_poly *p, int dst, int src) {
    p->x[dst] = p->x[src]; p->y[dst] = p->y[src];
    p->nx[dst] = p->nx[src]; p->ny[dst] = p->ny[src];
    p->id[dst] = p->id[src];
}

/* ConvexPolyhedron2::plane_cut (ConvexPolyhedron2.tcc:687-924) */
int or_poly_plane_cut(or_poly *p, double ox, double oy, double nx, double ny, int64_t cut_id, int normalized) {
    const int n = p->n;
    int nb_out = 0, first_out = -1;
    for (int i = 0; i < n; ++i) {
        double d = (ox - p->x[i]) * nx + (oy - p->y[i]) * ny;
        p->dist[i] = d;
        p->out[i] = d < 0;
        if (d < 0) {
            ++nb_out;
            if (first_out < 0) first_out = i;
        }
    }
    if (nb_out == 0) return 0;
    if (nb_out == n) {
        p->n = 0;
        return 0;
    }
    if (!normalized) {
        double s = 1 / sqrt(nx * nx + ny * ny);
        for (int i = 0; i < n; ++i) p->dist[i] *= s;
        nx *= s;
        ny *= s;
    }
    const double *D = p->dist;
    int i1 = first_out;
    if (nb_out == 1) {
        int i0 = (i1 + n - 1) % n, i2 = (i1 + 1) % n;
        double p0x = p->x[i0], p0y = p->y[i0], p1x = p->x[i1], p1y = p->y[i1], p2x = p->x[i2], p2y = p->y[i2];
        double s0 = D[i0], s1 = D[i1], s2 = D[i2];
        double m0 = s0 / (s1 - s0), m1 = s2 / (s1 - s2);
        poly_reserve(p, n + 1);
        p->n = n + 1;
        for (int i = n; i > i1 + 1; --i) mv(p, i, i - 1);
        p->x[i1 + 1] = p2x - m1 * (p1x - p2x);
        p->y[i1 + 1] = p2y - m1 * (p1y - p2y);
        p->id[i1 + 1] = p->id[i1];
        p->nx[i1 + 1] = p->nx[i1];
        p->ny[i1 + 1] = p->ny[i1];
        p->x[i1] = p0x - m0 * (p1x - p0x);
        p->y[i1] = p0y - m0 * (p1y - p0y);
        p->id[i1] = cut_id;
        p->nx[i1] = nx;
        p->ny[i1] = ny;
        return 1;
    }
    if (nb_out == 2) {
        if (i1 == 0 && !p->out[1]) i1 = n - 1;
        int i0 = (i1 + n - 1) % n, i2 = (i1 + 1) % n, i3 = (i1 + 2) % n;
        double p0x = p->x[i0], p0y = p->y[i0], p1x = p->x[i1], p1y = p->y[i1];
        double p2x = p->x[i2], p2y = p->y[i2], p3x = p->x[i3], p3y = p->y[i3];
        double m1 = D[i0] / (D[i1] - D[i0]), m2 = D[i3] / (D[i2] - D[i3]);
        p->x[i1] = p0x - m1 * (p1x - p0x);
        p->y[i1] = p0y - m1 * (p1y - p0y);
        p->id[i1] = cut_id;
        p->nx[i1] = nx;
        p->ny[i1] = ny;
        p->x[i2] = p3x - m2 * (p2x - p3x);
        p->y[i2] = p3y - m2 * (p2y - p3y);
        return 1;
    }
    if (i1 == 0 && p->out[n - 1]) {
        int nb_in = n - nb_out, i3 = 0;
        while (p->out[i3]) ++i3;
        i1 = nb_in + i3;
        int i0 = i1 - 1, i2 = i3 - 1;
        double p0x = p->x[i0], p0y = p->y[i0], p1x = p->x[i1], p1y = p->y[i1];
        double p2x = p->x[i2], p2y = p->y[i2], p3x = p->x[i3], p3y = p->y[i3];
        double m1 = D[i0] / (D[i1] - D[i0]), m2 = D[i3] / (D[i2] - D[i3]);
        p->x[0] = p3x - m2 * (p2x - p3x);
        p->y[0] = p3y - m2 * (p2y - p3y);
        p->id[0] = p->id[i2];
        p->nx[0] = p->nx[i2];
        p->ny[0] = p->ny[i2];
        int o = 1;
        for (; o <= nb_in; ++o) mv(p, o, i2 + o);
        p->x[o] = p0x - m1 * (p1x - p0x);
        p->y[o] = p0y - m1 * (p1y - p0y);
        p->id[o] = cut_id;
        p->nx[o] = nx;
        p->ny[o] = ny;
        p->n = n - nb_out + 2;
        return 1;
    }
    {
        int i0 = (i1 + n - 1) % n, i2 = (i1 + nb_out - 1) % n, i3 = (i1 + nb_out) % n;
        double p0x = p->x[i0], p0y = p->y[i0], p1x = p->x[i1], p1y = p->y[i1];
        double p2x = p->x[i2], p2y = p->y[i2], p3x = p->x[i3], p3y = p->y[i3];
        double m1 = D[i0] / (D[i1] - D[i0]), m2 = D[i3] / (D[i2] - D[i3]);
        p->x[i1] = p0x - m1 * (p1x - p0x);
        p->y[i1] = p0y - m1 * (p1y - p0y);
        p->id[i1] = cut_id;
        p->nx[i1] = nx;
        p->ny[i1] = ny;
        p->x[i1 + 1] = p3x - m2 * (p2x - p3x);
        p->y[i1 + 1] = p3y - m2 * (p2y - p3y);
        p->id[i1 + 1] = p->id[i2];
        p->nx[i1 + 1] = p->nx[i2];
        p->ny[i1 + 1] = p->ny[i2];
        int nb_rem = nb_out - 2;
        for (int i = i2 + 1; i < n; ++i) mv(p, i - nb_rem, i);
        p->n = n - nb_rem;
        return 1;
    }
}

/* ---------------------------------------------------------------- ball cut */
typedef struct { int type; int64_t id; double nx, ny, x, y; } TmpCut;

static void unique_inter(double cx, double cy, double r, double p0x, double p0y, double p1x, double p1y,
                         double *ox, double *oy) {
    double dx = p1x - p0x, dy = p1y - p0y;
    double a = dx * dx + dy * dy;
    double b = (p0x - cx) * dx + (p0y - cy) * dy;
    double c = (p0x - cx) * (p0x - cx) + (p0y - cy) * (p0y - cy) - r * r;
    double d = sqrt(fmax(0.0, b * b - a * c));
    double u = (-b + d) / a, v = (-b - d) / a;
    double t = fabs(u - 0.5) <= fabs(v - 0.5) ? u : v;
    t = fmin(1.0, fmax(0.0, t));
    *ox = p0x + t * dx;
    *oy = p0y + t * dy;
}

static int two_cuts(double cx, double cy, double r, double p0x, double p0y, double p1x, double p1y, double *ax,
                    double *ay, double *bx, double *by) {
    double dx = p1x - p0x, dy = p1y - p0y;
    double a = dx * dx + dy * dy;
    if (a == 0) return 0;
    double b = (p0x - cx) * dx + (p0y - cy) * dy;
    double c = (p0x - cx) * (p0x - cx) + (p0y - cy) * (p0y - cy) - r * r;
    double s = b * b - a * c;
    if (s <= 0) return 0;
    double d = sqrt(s);
    double u = (-b - d) / a, v = (-b + d) / a;
    if (u > 0 && u < 1)
        v = fmax(0.0, fmin(1.0, v));
    else if (v > 0 && v < 1)
        u = fmax(0.0, fmin(1.0, u));
    else
        return 0;
    *ax = p0x + u * dx; *ay = p0y + u * dy;
    *bx = p0x + v * dx; *by = p0y + v * dy;
    return atan2(*ay - cy, *ax - cx) != atan2(*by - cy, *bx - cx);
}

/* ConvexPolyhedron2::ball_cut (ConvexPolyhedron2.tcc:534-666) */
void or_poly_ball_cut(or_poly *p, double cx, double cy, double r, int64_t cut_id) {
    p->scx = cx; p->scy = cy; p->sr = r; p->sid = cut_id;
    const int n = p->n;
    if (n == 0) {
        p->sr = 0;
        return;
    }
    int all_inside = 1;
    for (int i = 0; i < n; ++i) {
        double d = (p->x[i] - cx) * (p->x[i] - cx) + (p->y[i] - cy) * (p->y[i] - cy) - r * r;
        p->dist[i] = d;
        all_inside &= d <= 0;
    }
    if (all_inside) return;
    TmpCut *tc = malloc(sizeof(TmpCut) * (2 * n + 2));
    int nt = 0;
    for (int e = 0; e < n; ++e) {
        int i0 = e == n - 1 ? n - 1 : e, i1 = e == n - 1 ? 0 : e + 1;
        double p0x = p->x[i0], p0y = p->y[i0], p1x = p->x[i1], p1y = p->y[i1];
        if (p->dist[i0] <= 0) {
            if (p->dist[i1] <= 0) {
                tc[nt++] = (TmpCut){LINE, p->id[i0], p->nx[i0], p->ny[i0], p0x, p0y};
            } else {
                double ix, iy;
                unique_inter(cx, cy, r, p0x, p0y, p1x, p1y, &ix, &iy);
                tc[nt++] = (TmpCut){LINE, p->id[i0], p->nx[i0], p->ny[i0], p0x, p0y};
                tc[nt++] = (TmpCut){ARC, cut_id, 0, 0, ix, iy};
            }
        } else {
            if (p->dist[i1] <= 0) {
                double ix, iy;
                unique_inter(cx, cy, r, p1x, p1y, p0x, p0y, &ix, &iy);
                tc[nt++] = (TmpCut){LINE, p->id[i0], p->nx[i0], p->ny[i0], ix, iy};
            } else {
                double ax, ay, bx, by;
                if (two_cuts(cx, cy, r, p0x, p0y, p1x, p1y, &ax, &ay, &bx, &by)) {
                    tc[nt++] = (TmpCut){LINE, p->id[i0], p->nx[i0], p->ny[i0], ax, ay};
                    tc[nt++] = (TmpCut){ARC, cut_id, 0, 0, bx, by};
                }
            }
        }
    }
    if (nt == 0) {
        for (int i0 = 0; i0 < n; ++i0)
            if ((cx - p->x[i0]) * p->nx[i0] + (cy - p->y[i0]) * p->ny[i0] > 0) {
                p->sr = 0;
                break;
            }
    }
    poly_reserve(p, nt);
    p->n = nt;
    for (int i = 0; i < nt; ++i) {
        p->x[i] = tc[i].x; p->y[i] = tc[i].y;
        p->nx[i] = tc[i].nx; p->ny[i] = tc[i].ny;
        p->id[i] = tc[i].id;
        p->arc[i] = (unsigned char)tc[i].type;
    }
    free(tc);
}

/* ConvexPolyhedron2::intersect_with (ConvexPolyhedron2.tcc:2475-2496) */
void or_poly_intersect_with(or_poly *p, const or_poly *q) {
    if (q->n) {
        for (int i = 0; i < q->n; ++i) or_poly_plane_cut(p, q->x[i], q->y[i], q->nx[i], q->ny[i], q->id[i], 1);
        if (q->sr > 0)
            or_poly_ball_cut(p, q->scx, q->scy, q->sr, q->sid);
        else {
            p->scx = q->scx; p->scy = q->scy; p->sr = q->sr; p->sid = q->sid;
        }
    } else {
        if (q->sr > 0)
            or_poly_ball_cut(p, q->scx, q->scy, q->sr, q->sid);
        else {
            p->sr = -1;
            p->n = 0;
        }
    }
}

/* ------------------------------------------------------------ integrals */
static double arc_angles(const or_poly *p, double p0x, double p0y, double p1x, double p1y, double *a0) {
    *a0 = atan2(p0y - p->scy, p0x - p->scx);
    double a1 = atan2(p1y - p->scy, p1x - p->scx);
    if (a1 < *a0) a1 += 2 * M_PI;
    return a1;
}

/* _arc_area (ConvexPolyhedron2.tcc:2361-2381) */
static double arc_area(const or_poly *p, double p0x, double p0y, double p1x, double p1y) {
    double a0, a1 = arc_angles(p, p0x, p0y, p1x, p1y, &a0);
    double ex = p0x - p1x, ey = p0y - p1y;
    double d0 = sqrt(ex * ex + ey * ey) / 2;
    double d1 = sqrt(fmax(0.0, p->sr * p->sr - d0 * d0));
    double rs = p->sr * p->sr * (a1 - a0) / 2;
    return a1 - a0 > M_PI ? rs + d1 * d0 : rs - d1 * d0;
}

/* integration( Constant, Unit ) (ConvexPolyhedron2.tcc:1791-1843), coeff 1 */
double or_poly_measure(const or_poly *p) {
    if (p->n == 0) return p->sr > 0 ? M_PI * p->sr * p->sr : 0.0;
    double res = 0;
    for (int i = 2; i < p->n; ++i) {
        double ax = p->x[0], ay = p->y[0], bx = p->x[i - 1], by = p->y[i - 1], cx = p->x[i], cy = p->y[i];
        res += ax * (by - cy) + bx * (cy - ay) + cx * (ay - by);
    }
    res *= 0.5;
    for (int i1 = 0, i0 = p->n - 1; i1 < p->n; i0 = i1++)
        if (p->arc[i0]) res += arc_area(p, p->x[i0], p->y[i0], p->x[i1], p->y[i1]);
    return res;
}

/* _centroid_arc (ConvexPolyhedron2.tcc:2296-2334) */
static void centroid_arc(const or_poly *p, double *ctd, double *mea, double p0x, double p0y, double p1x, double p1y,
                         double coeff) {
    double r = p->sr;
    p0x -= p->scx; p0y -= p->scy;
    p1x -= p->scx; p1y -= p->scy;
    double a0 = atan2(p0y, p0x), a1 = atan2(p1y, p1x);
    if (a1 < a0) a1 += 2 * M_PI;
    double ex = p0x - p1x, ey = p0y - p1y;
    double d0 = sqrt(ex * ex + ey * ey) / 2;
    double d1 = sqrt(fmax(0.0, r * r - d0 * d0));
    double tri_area = d1 * d0;
    double tbx = (1.0 / 3) * (p0x + p1x), tby = (1.0 / 3) * (p0y + p1y);
    double pie_area = r * r * (a1 - a0) / 2;
    double f = 2.0 / 3 * pow(r, 3) * sin((a1 - a0) / 2);
    double pmx = f * cos((a1 + a0) / 2), pmy = f * sin((a1 + a0) / 2);
    double lea;
    if (a1 - a0 > M_PI) {
        ctd[0] += coeff * (pmx + tri_area * tbx);
        ctd[1] += coeff * (pmy + tri_area * tby);
        lea = (pie_area + tri_area) * coeff;
    } else {
        ctd[0] += coeff * (pmx - tri_area * tbx);
        ctd[1] += coeff * (pmy - tri_area * tby);
        lea = (pie_area - tri_area) * coeff;
    }
    ctd[0] += lea * p->scx;
    ctd[1] += lea * p->scy;
    *mea += lea;
}

/* add_centroid_contrib( Constant, Unit ) (ConvexPolyhedron2.tcc:1047-1074) */
static void centroid_contrib(const or_poly *p, double coeff, double *ctd, double *mea) {
    if (p->n == 0) {
        if (p->sr >= 0) {
            double lea = M_PI * p->sr * p->sr * coeff;
            ctd[0] += lea * p->scx;
            ctd[1] += lea * p->scy;
            *mea += lea;
        }
        return;
    }
    for (int i = 2; i < p->n; ++i) {
        double ax = p->x[0], ay = p->y[0], bx = p->x[i - 1], by = p->y[i - 1], cx = p->x[i], cy = p->y[i];
        double lea = 0.5 * (ax * (by - cy) + bx * (cy - ay) + cx * (ay - by)) * coeff;
        double f = (1.0 / 3) * lea;
        ctd[0] += f * (ax + bx + cx);
        ctd[1] += f * (ay + by + cy);
        *mea += lea;
    }
    for (int i1 = 0, i0 = p->n - 1; i1 < p->n; i0 = i1++)
        if (p->arc[i0]) centroid_arc(p, ctd, mea, p->x[i0], p->y[i0], p->x[i1], p->y[i1], coeff);
}

void or_poly_centroid(const or_poly *p, double coeff, double *ctd2, double *mass) {
    double c[2] = {0, 0}, m = 0;
    centroid_contrib(p, coeff, c, &m);
    double d = m + (m == 0);
    ctd2[0] = c[0] / d;
    ctd2[1] = c[1] / d;
    if (mass) *mass = m;
}

/* integral over each fan triangle of c0 + c1 x + c2 y + c3 x^2 + c4 xy + c5 y^2
 * by the exact triangle moments (same quantity as ConvexPolyhedron2.tcc:2181-2225) */
double or_poly_integrate_poly6(const or_poly *p, const double *c) {
    double res = 0;
    for (int i = 2; i < p->n; ++i) {
        double ax = p->x[0], ay = p->y[0], bx = p->x[i - 1], by = p->y[i - 1], cx = p->x[i], cy = p->y[i];
        double s = 0.5 * (ax * (by - cy) + bx * (cy - ay) + cx * (ay - by));
        double mx = (ax + bx + cx) / 3, my = (ay + by + cy) / 3;
        double xx = (ax * ax + bx * bx + cx * cx + ax * bx + ax * cx + bx * cx) / 6;
        double yy = (ay * ay + by * by + cy * cy + ay * by + ay * cy + by * cy) / 6;
        double xy = (2 * ax * ay + 2 * bx * by + 2 * cx * cy + ax * by + ay * bx + ax * cy + ay * cx + bx * cy + by * cx) / 12;
        res += s * (c[0] + c[1] * mx + c[2] * my + c[3] * xx + c[4] * xy + c[5] * yy);
    }
    return res;
}

static double poly6_at(const double *c, double x, double y) {
    return c[0] + c[1] * x + c[2] * y + c[3] * x * x + c[4] * x * y + c[5] * y * y;
}

/* first moments (integrals of x f and y f) of the same density over the fan
 * triangles, by the 7-point triangle rule (weights 1/20 at the vertices, 2/15
 * at the edge midpoints, 9/20 at the centroid, times the area), exact for
 * cubics: the quantity of add_centroid_contrib( Polynomial<6>, Unit )
 * (ConvexPolyhedron2.tcc:980-1044) */
static void poly6_moments(const or_poly *p, const double *c, double *mom) {
    for (int i = 2; i < p->n; ++i) {
        double v[3][2] = {{p->x[0], p->y[0]}, {p->x[i - 1], p->y[i - 1]}, {p->x[i], p->y[i]}};
        double a = 0.5 * (v[0][0] * (v[1][1] - v[2][1]) + v[1][0] * (v[2][1] - v[0][1]) + v[2][0] * (v[0][1] - v[1][1]));
        double sx = 0, sy = 0;
        for (int k = 0; k < 3; ++k) {
            double fv = poly6_at(c, v[k][0], v[k][1]);
            double mx = 0.5 * (v[k][0] + v[(k + 1) % 3][0]), my = 0.5 * (v[k][1] + v[(k + 1) % 3][1]);
            double fm = poly6_at(c, mx, my);
            sx += (1.0 / 20.0) * v[k][0] * fv + (2.0 / 15.0) * mx * fm;
            sy += (1.0 / 20.0) * v[k][1] * fv + (2.0 / 15.0) * my * fm;
        }
        double gx = (v[0][0] + v[1][0] + v[2][0]) / 3, gy = (v[0][1] + v[1][1] + v[2][1]) / 3;
        double fg = poly6_at(c, gx, gy);
        mom[0] += a * (sx + (9.0 / 20.0) * gx * fg);
        mom[1] += a * (sy + (9.0 / 20.0) * gy * fg);
    }
}

static void min_max_position(const or_poly *p, double *mn, double *mx) {
    mn[0] = mn[1] = DBL_MAX;
    mx[0] = mx[1] = -DBL_MAX;
    if (p->n == 0 && p->sr > 0) { /* full disc: the disc's bounding box */
        mn[0] = p->scx - p->sr; mn[1] = p->scy - p->sr;
        mx[0] = p->scx + p->sr; mx[1] = p->scy + p->sr;
        return;
    }
    for (int i = 0; i < p->n; ++i) {
        if (p->arc[i]) {
            mn[0] = fmin(mn[0], p->scx - p->sr); mn[1] = fmin(mn[1], p->scy - p->sr);
            mx[0] = fmax(mx[0], p->scx + p->sr); mx[1] = fmax(mx[1], p->scy + p->sr);
        } else {
            mn[0] = fmin(mn[0], p->x[i]); mn[1] = fmin(mn[1], p->y[i]);
            mx[0] = fmax(mx[0], p->x[i]); mx[1] = fmax(mx[1], p->y[i]);
        }
    }
}

/* ------------------------------------------------------------- domain */
typedef struct { or_poly *poly; double coeff; } Item;

struct or_domain {
    int nitems, cap;
    Item *items;
    int image;
    double img_lo[2], img_hi[2];
    int64_t sizes[2];
    int nb_coeffs;
    double *data;
    or_poly *englobing;
};

or_domain *or_domain_new(void) { return calloc(1, sizeof(or_domain)); }

void or_domain_free(or_domain *d) {
    if (!d) return;
    for (int i = 0; i < d->nitems; ++i) or_poly_free(d->items[i].poly);
    free(d->items);
    free(d->data);
    or_poly_free(d->englobing);
    free(d);
}

static void add_item(or_domain *d, or_poly *p, double coeff) {
    if (d->nitems == d->cap) {
        d->cap = d->cap ? 2 * d->cap : 4;
        d->items = realloc(d->items, d->cap * sizeof(Item));
    }
    d->items[d->nitems++] = (Item){p, coeff};
    or_poly_free(d->englobing);
    d->englobing = NULL;
}

/* ConvexPolyhedronAssembly::add_box (ConvexPolyhedronAssembly.tcc:46-50) */
void or_domain_add_box(or_domain *d, const double *p0, const double *p1, double coeff) {
    add_item(d, or_poly_box(p0[0], p0[1], p1[0], p1[1], -1), coeff);
}

void or_domain_add_simplex(or_domain *d, const double *pts6, double coeff) {
    add_item(d, or_poly_simplex(pts6, -1), coeff);
}

/* ConvexPolyhedronAssembly::add_convex_polyhedron (ConvexPolyhedronAssembly.tcc:7-33) */
void or_domain_add_convex_polyhedron(or_domain *d, const double *pts, const double *nrm, int64_t m, double coeff) {
    double mn[2], mx[2], de[2];
    for (int k = 0; k < 2; ++k) {
        mn[k] = DBL_MAX;
        mx[k] = -DBL_MAX;
        for (int64_t i = 0; i < m; ++i) {
            mn[k] = fmin(mn[k], pts[2 * i + k]);
            mx[k] = fmax(mx[k], pts[2 * i + k]);
        }
        de[k] = mx[k] - mn[k];
    }
    or_poly *p = or_poly_box(mn[0] - de[0], mn[1] - de[1], mx[0] + de[0], mx[1] + de[1], -1);
    for (int64_t i = 0; i < m; ++i) {
        double nx = nrm[2 * i], ny = nrm[2 * i + 1];
        double l = sqrt(nx * nx + ny * ny) + 1e-40; /* Point2 normalized() */
        or_poly_plane_cut(p, pts[2 * i], pts[2 * i + 1], nx / l, ny / l, -1, 1);
    }
    add_item(d, p, coeff);
}

void or_domain_set_image(or_domain *d, const double *min_pt, const double *max_pt, const double *data,
                         const int64_t *sizes, int nb_coeffs) {
    d->image = 1;
    for (int k = 0; k < 2; ++k) {
        d->img_lo[k] = min_pt[k];
        d->img_hi[k] = max_pt[k];
        d->sizes[k] = sizes[k];
    }
    d->nb_coeffs = nb_coeffs;
    size_t cnt = (size_t)sizes[0] * sizes[1] * nb_coeffs;
    free(d->data);
    d->data = malloc(cnt * sizeof(double));
    memcpy(d->data, data, cnt * sizeof(double));
    or_poly_free(d->englobing);
    d->englobing = or_poly_box(min_pt[0], min_pt[1], max_pt[0], max_pt[1], -1);
}

/* ConvexPolyhedronAssembly::measure (:115-120) and ScaledImage::measure (ScaledImage.tcc:36-69) */
double or_domain_measure(const or_domain *d) {
    if (d->image) {
        int64_t np = d->sizes[0] * d->sizes[1];
        double res = 0;
        if (d->nb_coeffs == 1) {
            for (int64_t i = 0; i < np; ++i) res += d->data[i];
            res /= np;
        } else {
            double psx = (d->img_hi[0] - d->img_lo[0]) / d->sizes[0], psy = (d->img_hi[1] - d->img_lo[1]) / d->sizes[1];
            for (int64_t yi = 0; yi < d->sizes[1]; ++yi)
                for (int64_t xi = 0; xi < d->sizes[0]; ++xi) {
                    or_poly *px = or_poly_box(d->img_lo[0] + psx * xi, d->img_lo[1] + psy * yi,
                                              d->img_lo[0] + psx * (xi + 1), d->img_lo[1] + psy * (yi + 1), -1);
                    double c[6];
                    for (int k = 0; k < 6; ++k) c[k] = d->data[np * k + yi * d->sizes[0] + xi];
                    res += or_poly_integrate_poly6(px, c) / (psx * psy);
                    or_poly_free(px);
                }
            res /= np;
        }
        return res * (d->img_hi[0] - d->img_lo[0]) * (d->img_hi[1] - d->img_lo[1]);
    }
    double res = 0;
    for (int i = 0; i < d->nitems; ++i) res += d->items[i].coeff * or_poly_measure(d->items[i].poly);
    return res;
}

/* ConvexPolyhedronAssembly::normalize (:53-57) */
void or_domain_normalize(or_domain *d) {
    double m = or_domain_measure(d);
    if (m == 0) return;
    if (d->image) {
        int64_t cnt = d->sizes[0] * d->sizes[1] * d->nb_coeffs;
        for (int64_t i = 0; i < cnt; ++i) d->data[i] /= m;
    } else {
        for (int i = 0; i < d->nitems; ++i) d->items[i].coeff /= m;
    }
}

/* ConvexPolyhedronAssembly::englobing_convex_polyhedron (:60-92) */
static const or_poly *englobing(or_domain *d) {
    if (d->image) return d->englobing;
    if (d->nitems == 1) return d->items[0].poly;
    if (!d->englobing) {
        double mn[2] = {DBL_MAX, DBL_MAX}, mx[2] = {-DBL_MAX, -DBL_MAX};
        for (int i = 0; i < d->nitems; ++i) {
            double a[2], b[2];
            min_max_position(d->items[i].poly, a, b);
            for (int k = 0; k < 2; ++k) { mn[k] = fmin(mn[k], a[k]); mx[k] = fmax(mx[k], b[k]); }
        }
        double de[2] = {mx[0] - mn[0], mx[1] - mn[1]};
        d->englobing = or_poly_box(mn[0] - de[0], mn[1] - de[1], mx[0] + de[0], mx[1] + de[1], -1);
    }
    return d->englobing;
}

/* -------------------------------------------------------- cell callback */
typedef struct { int64_t col; double val; } RowItem;

typedef struct {
    int64_t n, i;
    const double *pos;
    double w0;
    double mass, mass_c, ctd[2], der0;
    RowItem *items;
    int nitems, cap_items;
} CellAcc;

static void push_item(CellAcc *a, int64_t c, double v) {
    if (a->nitems == a->cap_items) {
        a->cap_items = a->cap_items ? 2 * a->cap_items : 32;
        a->items = realloc(a->items, a->cap_items * sizeof(RowItem));
    }
    a->items[a->nitems++] = (RowItem){c, v};
}

/* get_der_integrals_wrt_weights' per-piece callback (get_der_integrals_wrt_weights.h:51-74)
 * with for_each_boundary_item( Constant, Unit ) (ConvexPolyhedron2.tcc:437-478) */
static void piece(CellAcc *a, const or_poly *cp, int is_poly6, const double *c6, double coeff) {
    if (is_poly6) {
        const double m6 = or_poly_integrate_poly6(cp, c6);
        a->mass += m6;
        a->mass_c += m6;
        poly6_moments(cp, c6, a->ctd);
    } else {
        a->mass += coeff * or_poly_measure(cp);
        centroid_contrib(cp, coeff, a->ctd, &a->mass_c);
    }
    const double x0 = a->pos[2 * a->i], y0 = a->pos[2 * a->i + 1];
    if (cp->n == 0) {
        if (cp->sr >= 0) {
            double m = coeff * 2 * M_PI * cp->sr;
            if (cp->sid == a->i) a->der0 += 0.5 * m / sqrt(a->w0);
        }
        return;
    }
    for (int i1 = 0, i0 = cp->n - 1; i1 < cp->n; i0 = i1++) {
        double m;
        if (cp->arc[i0]) {
            double a0, a1 = arc_angles(cp, cp->x[i0], cp->y[i0], cp->x[i1], cp->y[i1], &a0);
            m = coeff * (a1 - a0) * cp->sr;
        } else {
            double dx = cp->x[i1] - cp->x[i0], dy = cp->y[i1] - cp->y[i0];
            m = coeff * sqrt(dx * dx + dy * dy);
            if (is_poly6) /* for_each_boundary_item( Polynomial<6>, Unit ) (:180-214): Simpson along the edge */
                m = sqrt(dx * dx + dy * dy) / 6.0 *
                    (poly6_at(c6, cp->x[i0], cp->y[i0]) +
                     4.0 * poly6_at(c6, 0.5 * (cp->x[i0] + cp->x[i1]), 0.5 * (cp->y[i0] + cp->y[i1])) +
                     poly6_at(c6, cp->x[i1], cp->y[i1]));
        }
        int64_t id = cp->id[i0];
        if (id == -1) continue;
        if (id == a->i) {
            a->der0 += 0.5 * m / sqrt(a->w0);
        } else {
            double dx = x0 - a->pos[2 * id], dy = y0 - a->pos[2 * id + 1];
            double dist = sqrt(dx * dx + dy * dy);
            if (dist) {
                double b = 0.5 * m / dist;
                push_item(a, id, -b);
                a->der0 += b;
            }
        }
    }
}

static int cmp_item(const void *pa, const void *pb) {
    const RowItem *a = pa, *b = pb;
    if (a->col != b->col) return a->col < b->col ? -1 : 1;
    return a->val < b->val ? -1 : (a->val > b->val ? 1 : 0);
}

/* bounds.for_each_intersection (ConvexPolyhedronAssembly.tcc:132-142, ScaledImage.tcc:98-149) */
static void for_each_intersection(or_domain *d, const or_poly *cell, or_poly *ccp, CellAcc *a) {
    if (d->image) {
        int64_t np = d->sizes[0] * d->sizes[1];
        if (np == 1) {
            piece(a, cell, d->nb_coeffs == 6, d->data, d->data[0]);
            return;
        }
        if (cell->n == 0 && !(cell->sr > 0)) return;
        double mn[2], mx[2], ps[2];
        int64_t lo[2], hi[2];
        min_max_position(cell, mn, mx);
        for (int k = 0; k < 2; ++k) {
            double mi = fmax(mn[k], d->img_lo[k]), ma = fmin(mx[k], d->img_hi[k]);
            int64_t a0 = (int64_t)((mi - d->img_lo[k]) * d->sizes[k] / (d->img_hi[k] - d->img_lo[k]));
            int64_t a1 = (int64_t)((ma - d->img_lo[k]) * d->sizes[k] / (d->img_hi[k] - d->img_lo[k]));
            if (a0 < 1) a0 = 1;
            lo[k] = a0 - 1;
            hi[k] = a1 + 2 < d->sizes[k] ? a1 + 2 : d->sizes[k];
            ps[k] = (d->img_hi[k] - d->img_lo[k]) / d->sizes[k];
        }
        for (int64_t yi = lo[1]; yi < hi[1]; ++yi)
            for (int64_t xi = lo[0]; xi < hi[0]; ++xi) {
                poly_box_into(ccp, d->img_lo[0] + ps[0] * (double)xi, d->img_lo[1] + ps[1] * (double)yi,
                              d->img_lo[0] + ps[0] * (double)(xi + 1), d->img_lo[1] + ps[1] * (double)(yi + 1), -1);
                or_poly_intersect_with(ccp, cell);
                int64_t pix = yi * d->sizes[0] + xi;
                if (d->nb_coeffs == 6) {
                    double c[6];
                    for (int k = 0; k < 6; ++k) c[k] = d->data[np * k + pix];
                    piece(a, ccp, 1, c, 0);
                } else {
                    piece(a, ccp, 0, NULL, d->data[pix]);
                }
            }
        return;
    }
    if (d->nitems == 1) {
        piece(a, cell, 0, NULL, d->items[0].coeff);
        return;
    }
    for (int it = 0; it < d->nitems; ++it) {
        poly_copy_into(ccp, d->items[it].poly);
        or_poly_intersect_with(ccp, cell);
        piece(a, ccp, 0, NULL, d->items[it].coeff);
    }
}

/* ------------------------------------------------------------- grid */
typedef struct {
    int64_t nx, ny;
    double lo[2], h[2];
    int64_t *start, *ind;
    double *maxw, *bmin, *bmax;
    double gmaxw;
} Grid;

static void grid_build(Grid *g, int64_t n, const double *pos, const double *w) {
    double lo[2] = {DBL_MAX, DBL_MAX}, hi[2] = {-DBL_MAX, -DBL_MAX};
    g->gmaxw = -DBL_MAX;
    for (int64_t i = 0; i < n; ++i) {
        for (int k = 0; k < 2; ++k) {
            lo[k] = fmin(lo[k], pos[2 * i + k]);
            hi[k] = fmax(hi[k], pos[2 * i + k]);
        }
        g->gmaxw = fmax(g->gmaxw, w[i]);
    }
    int64_t side = (int64_t)ceil(sqrt((double)n / 2.0));
    if (side < 1) side = 1;
    g->nx = g->ny = side;
    for (int k = 0; k < 2; ++k) {
        g->lo[k] = lo[k];
        double e = hi[k] - lo[k];
        g->h[k] = e > 0 ? e / side * (1 + 1e-12) : 1.0;
    }
    int64_t nc = g->nx * g->ny;
    g->start = calloc(nc + 1, sizeof(int64_t));
    g->ind = malloc((n ? n : 1) * sizeof(int64_t));
    g->maxw = malloc(nc * sizeof(double));
    g->bmin = malloc(2 * nc * sizeof(double));
    g->bmax = malloc(2 * nc * sizeof(double));
    int64_t *cell = malloc((n ? n : 1) * sizeof(int64_t));
    for (int64_t i = 0; i < n; ++i) {
        int64_t cx = (int64_t)((pos[2 * i] - g->lo[0]) / g->h[0]);
        int64_t cy = (int64_t)((pos[2 * i + 1] - g->lo[1]) / g->h[1]);
        if (cx >= g->nx) cx = g->nx - 1;
        if (cy >= g->ny) cy = g->ny - 1;
        cell[i] = cy * g->nx + cx;
        g->start[cell[i] + 1]++;
    }
    for (int64_t c = 0; c < nc; ++c) g->start[c + 1] += g->start[c];
    int64_t *fill = malloc(nc * sizeof(int64_t));
    memcpy(fill, g->start, nc * sizeof(int64_t));
    for (int64_t i = 0; i < n; ++i) g->ind[fill[cell[i]]++] = i;
    for (int64_t c = 0; c < nc; ++c) {
        g->maxw[c] = -DBL_MAX;
        g->bmin[2 * c] = g->bmin[2 * c + 1] = DBL_MAX;
        g->bmax[2 * c] = g->bmax[2 * c + 1] = -DBL_MAX;
        for (int64_t k = g->start[c]; k < g->start[c + 1]; ++k) {
            int64_t i = g->ind[k];
            g->maxw[c] = fmax(g->maxw[c], w[i]);
            for (int d = 0; d < 2; ++d) {
                g->bmin[2 * c + d] = fmin(g->bmin[2 * c + d], pos[2 * i + d]);
                g->bmax[2 * c + d] = fmax(g->bmax[2 * c + d], pos[2 * i + d]);
            }
        }
    }
    free(fill);
    free(cell);
}

static void grid_free(Grid *g) {
    free(g->start); free(g->ind); free(g->maxw); free(g->bmin); free(g->bmax);
}

/* SpZGrid::can_be_evicted, active branch (SpZGrid.tcc:475-480) */
static int can_be_evicted(const or_poly *lc, double c0x, double c0y, double w0, const double *bmin, const double *bmax,
                          double maxw) {
    for (int k = 0; k < lc->n; ++k) {
        double px = lc->x[k], py = lc->y[k];
        double qx = fmin(bmax[0], fmax(bmin[0], px)), qy = fmin(bmax[1], fmax(bmin[1], py));
        if (!((c0x - px) * (c0x - px) + (c0y - py) * (c0y - py) - w0 <= (qx - px) * (qx - px) + (qy - py) * (qy - py) - maxw))
            return 0;
    }
    return 1;
}

/* no Dirac outside the square of rings < R around the home cell can cut:
 * for every vertex p, |c0 - p|^2 - w0 <= dist(p, outside)^2 - max weight */
static int rings_done(const or_poly *lc, const Grid *g, int64_t hx, int64_t hy, int64_t R, double c0x, double c0y,
                      double w0) {
    double x0 = g->lo[0] + (hx - (R - 1)) * g->h[0], x1 = g->lo[0] + (hx + R) * g->h[0];
    double y0 = g->lo[1] + (hy - (R - 1)) * g->h[1], y1 = g->lo[1] + (hy + R) * g->h[1];
    int cover = hx - (R - 1) <= 0 && hy - (R - 1) <= 0 && hx + R >= g->nx && hy + R >= g->ny;
    if (cover) return 1;
    for (int k = 0; k < lc->n; ++k) {
        double px = lc->x[k], py = lc->y[k];
        double d = 0;
        if (px > x0 && px < x1 && py > y0 && py < y1) {
            d = px - x0;
            d = fmin(d, x1 - px);
            d = fmin(d, py - y0);
            d = fmin(d, y1 - py);
        }
        double lhs = (c0x - px) * (c0x - px) + (c0y - py) * (c0y - py) - w0;
        if (!(lhs <= d * d - g->gmaxw)) return 0;
    }
    return 1;
}

static void cut_with_cell(or_poly *lc, const Grid *g, int64_t c, int64_t i, const double *pos, const double *w) {
    const double c0x = pos[2 * i], c0y = pos[2 * i + 1], w0 = w[i];
    for (int64_t k = g->start[c]; k < g->start[c + 1]; ++k) {
        int64_t j = g->ind[k];
        if (j == i) continue;
        /* SpZGrid.tcc:506-522 */
        double vx = pos[2 * j] - c0x, vy = pos[2 * j + 1] - c0y;
        double nn = vx * vx + vy * vy;
        double x = 0.5 + 0.5 * (w0 - w[j]) / nn;
        or_poly_plane_cut(lc, c0x + x * vx, c0y + x * vy, vx, vy, j, 0);
        if (lc->n == 0) return;
    }
}

static void build_cell(or_poly *lc, const or_poly *start, const Grid *g, int64_t i, const double *pos, const double *w) {
    poly_copy_into(lc, start);
    const double c0x = pos[2 * i], c0y = pos[2 * i + 1], w0 = w[i];
    int64_t hx = (int64_t)((c0x - g->lo[0]) / g->h[0]), hy = (int64_t)((c0y - g->lo[1]) / g->h[1]);
    if (hx >= g->nx) hx = g->nx - 1;
    if (hy >= g->ny) hy = g->ny - 1;
    for (int64_t R = 0;; ++R) {
        if (R > 0 && rings_done(lc, g, hx, hy, R, c0x, c0y, w0)) break;
        if (R > g->nx + g->ny) break;
        for (int64_t cy = hy - R; cy <= hy + R; ++cy) {
            if (cy < 0 || cy >= g->ny) continue;
            for (int64_t cx = hx - R; cx <= hx + R; ++cx) {
                if (cx < 0 || cx >= g->nx) continue;
                if (cy != hy - R && cy != hy + R && cx != hx - R && cx != hx + R) continue;
                int64_t c = cy * g->nx + cx;
                if (g->start[c] == g->start[c + 1]) continue;
                if (lc->n == 0) return;
                if (can_be_evicted(lc, c0x, c0y, w0, g->bmin + 2 * c, g->bmax + 2 * c, g->maxw[c])) continue;
                cut_with_cell(lc, g, c, i, pos, w);
            }
        }
        if (lc->n == 0) return;
    }
}

int or_power_diagram_2d(int64_t n, const double *pos, const double *w, const or_domain *dom_c, int ball_cut,
                        double *mass, double *ctd, double *mass_c, int64_t *offsets, int64_t *cols, double *vals,
                        int64_t csr_cap, int64_t *nb_off, int64_t *nb_ids, int64_t nb_cap) {
    or_domain *dom = (or_domain *)dom_c;
    const or_poly *start = englobing(dom);
    Grid g;
    grid_build(&g, n, pos, w);
    or_poly *lc = poly_new(), *ccp = poly_new();
    CellAcc a = {0};
    a.n = n;
    a.pos = pos;
    int64_t nnz = 0, nbt = 0;
    int status = 0;
    for (int64_t i = 0; i < n; ++i) {
        build_cell(lc, start, &g, i, pos, w);
        /* SpZGrid.tcc:633-636 */
        if (ball_cut)
            or_poly_ball_cut(lc, pos[2 * i], pos[2 * i + 1], sqrt(w[i]), i);
        else {
            lc->scx = pos[2 * i];
            lc->scy = pos[2 * i + 1];
        }
        if (nb_off) {
            nb_off[i] = nbt;
            for (int k = 0; k < lc->n; ++k) {
                if (nbt < nb_cap) nb_ids[nbt] = lc->arc[k] ? -2 : lc->id[k];
                ++nbt;
            }
        }
        a.i = i;
        a.w0 = w[i];
        a.mass = a.mass_c = a.der0 = 0;
        a.ctd[0] = a.ctd[1] = 0;
        a.nitems = 0;
        for_each_intersection(dom, lc, ccp, &a);
        if (mass) mass[i] = a.mass;
        if (mass_c) mass_c[i] = a.mass_c;
        if (ctd) {
            double d = a.mass_c + (a.mass_c == 0);
            ctd[2 * i] = a.ctd[0] / d;
            ctd[2 * i + 1] = a.ctd[1] / d;
        }
        if (offsets) {
            push_item(&a, i, a.der0);
            qsort(a.items, a.nitems, sizeof(RowItem), cmp_item);
            offsets[i] = nnz;
            for (int k = 0; k < a.nitems; ++k) {
                if (k + 1 < a.nitems && a.items[k].col == a.items[k + 1].col) {
                    a.items[k + 1].val += a.items[k].val;
                    continue;
                }
                if (nnz < csr_cap) {
                    cols[nnz] = a.items[k].col;
                    vals[nnz] = a.items[k].val;
                }
                ++nnz;
            }
        }
    }
    if (offsets) offsets[n] = nnz;
    if (nb_off) nb_off[n] = nbt;
    if (nnz > csr_cap || nbt > nb_cap) status = -1;
    free(a.items);
    or_poly_free(lc);
    or_poly_free(ccp);
    grid_free(&g);
    return status;
}
