/*
 * sdot_oracle.h -- CPU restatement of the reference's power-diagram path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the parity reference: tests/, the smoke test of
 * __graft_entry__ and bench.py's CPU-baseline leg may call it; the product
 * (sdot_b200/, libsdot_b200.so) never links or calls it.
 *
 * Plain C11, single-threaded, double precision, no fast-math.  Every
 * function cites the reference file:line it restates.
 */
#ifndef SDOT_ORACLE_H
#define SDOT_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- single polygon (ConvexPolyhedron2, 2D) -------------------------------- */
typedef struct or_poly or_poly;
or_poly *or_poly_box(double x0, double y0, double x1, double y1, int64_t cut_id);
or_poly *or_poly_simplex(const double *pts6, int64_t cut_id);
or_poly *or_poly_copy(const or_poly *p);
void or_poly_free(or_poly *p);
/* normalized != 0: the normal is used as given (N<1>); else distances are
 * divided by |normal| (N<0>).  Returns 1 on an effective cut.               */
int or_poly_plane_cut(or_poly *p, double ox, double oy, double nx, double ny, int64_t cut_id, int normalized);
void or_poly_ball_cut(or_poly *p, double cx, double cy, double r, int64_t cut_id);
void or_poly_intersect_with(or_poly *p, const or_poly *q);
int or_poly_nb_points(const or_poly *p);
void or_poly_points(const or_poly *p, double *xy, int64_t *ids, int *arcs);
double or_poly_measure(const or_poly *p);
/* centroid and mass with a constant density */
void or_poly_centroid(const or_poly *p, double coeff, double *ctd2, double *mass);
/* integral of c0 + c1 x + c2 y + c3 x^2 + c4 x y + c5 y^2 */
double or_poly_integrate_poly6(const or_poly *p, const double *c6);
double or_poly_sphere_radius(const or_poly *p);

/* ---- whole power diagram (2D) ------------------------------------------------
 * domain_kind: 0 = list of convex polygons (boxes / simplices / half-plane
 *   polyhedra, see or_domain_*), 1 = image.
 * Outputs (may be NULL): mass[n] (get_integrals), ctd[2n] and mass_c[n]
 * (get_centroids), Hessian CSR (offsets[n+1], cols[cap], vals[cap]) and
 * neighbour lists (nb_off[n+1], nb_ids[cap]).  Returns 0, or -1 when a CSR
 * or neighbour buffer is too small.                                          */
typedef struct or_domain or_domain;
or_domain *or_domain_new(void);
void or_domain_free(or_domain *d);
void or_domain_add_box(or_domain *d, const double *p0, const double *p1, double coeff);
void or_domain_add_simplex(or_domain *d, const double *pts6, double coeff);
void or_domain_add_convex_polyhedron(or_domain *d, const double *pts, const double *nrm, int64_t m, double coeff);
void or_domain_set_image(or_domain *d, const double *min_pt, const double *max_pt, const double *data,
                         const int64_t *sizes, int nb_coeffs);
void or_domain_normalize(or_domain *d);
double or_domain_measure(const or_domain *d);

int or_power_diagram_2d(int64_t n, const double *pos, const double *w, const or_domain *dom, int ball_cut,
                        double *mass, double *ctd, double *mass_c, int64_t *offsets, int64_t *cols, double *vals,
                        int64_t csr_cap, int64_t *nb_off, int64_t *nb_ids, int64_t nb_cap);

#ifdef __cplusplus
}
#endif
#endif
