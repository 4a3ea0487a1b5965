// C-ABI driver around the UNMODIFIED reference sdot headers.
//
// Test infrastructure only (the parity reference and the timed CPU baseline): it is
// compiled by oracle/Makefile, with the reference sources included from where
// they lie, into oracle/_ref/libsdot_ref.so.  Nothing in the product links it.
//
// It exposes the reference's own call sequence for the power-diagram path:
//   SpZGrid<Pc>::update                       (src/sdot/PowerDiagram/Visitors/SpZGrid.tcc:24-38)
//   get_integrals                             (src/sdot/PowerDiagram/get_integrals.h:12-21)
//   get_centroids                             (src/sdot/PowerDiagram/get_centroids.h:13-56)
//   get_der_integrals_wrt_weights             (src/sdot/PowerDiagram/get_der_integrals_wrt_weights.h:15-122)
// with ConvexPolyhedronAssembly (add_box / add_convex_polyhedron /
// add_simplex / normalize) or ScaledImage as bounds, and FunctionEnum::Unit or
// FunctionEnum::InBallW05 as the radial function.
//
// One deviation, documented: the ScaledImage bounds go through
// FixedScaledImage below, which restates ScaledImage::for_each_intersection
// (src/sdot/Domains/ScaledImage.tcc:98-149) with the pixel range of a
// vertex-free cell (a full disc) taken from the disc's bounding box.  The
// reference computes that range from ConvexPolyhedron2::min_position /
// max_position (ConvexPolyhedron2.tcc:502-524), which return +-DBL_MAX for a
// cell without vertices; the float->size_t conversion of that value is
// undefined behaviour and gives full discs a zero mass at -O3.
#include "src/sdot/Support/Stream.h"
#include "src/sdot/PowerDiagram/Visitors/SpZGrid.h"
#include "src/sdot/PowerDiagram/get_integrals.h"
#include "src/sdot/PowerDiagram/get_centroids.h"
#include "src/sdot/PowerDiagram/get_der_integrals_wrt_weights.h"
#include "src/sdot/PowerDiagram/get_image_integrals.h"
#include "src/sdot/PowerDiagram/get_image_of_cell_nums.h"
#include "src/sdot/PowerDiagram/get_der_centroids_and_integrals_wrt_weight_and_positions.h"
#include "src/sdot/Domains/ConvexPolyhedronAssembly.h"
#include "src/sdot/Domains/ScaledImage.h"
#include "src/sdot/Integration/Unit.h"
#include "src/sdot/Integration/InBallW05.h"
#include "src/sdot/Support/ThreadPool.h"

#include <chrono>
#include <cstdint>
#include <cstring>
#include <memory>
#include <vector>

using namespace sdot;

namespace {

// allow_translations = 1 compiles the traversal's periodic branch; with no
// translation set it takes the same path as allow_translations = 0
struct Pc2 { enum { dim = 2, allow_ball_cut = 1, allow_translations = 1 }; using TI = std::size_t; using TF = double; using CI = std::size_t; };
struct Pc3 { enum { dim = 3, allow_ball_cut = 0, allow_translations = 0 }; using TI = std::size_t; using TF = double; using CI = std::size_t; };

// ScaledImage::for_each_intersection with the full-disc bounding box fixed.
template <class Pc>
struct FixedScaledImage {
    static constexpr int dim = Pc::dim;
    using TF = typename Pc::TF;
    using TI = typename Pc::TI;
    using CP = typename std::conditional<dim == 3, ConvexPolyhedron3<Pc>, ConvexPolyhedron2<Pc>>::type;
    using Pt = typename CP::Pt;

    ScaledImage<Pc> img;
    Pt min_pt, max_pt;
    std::array<TI, dim> sizes;
    std::vector<TF> data;
    TI nb_coeffs;

    FixedScaledImage(Pt mi, Pt ma, const TF *d, std::array<TI, dim> s, TI nc)
        : img(mi, ma, d, s, nc), min_pt(mi), max_pt(ma), sizes(s), nb_coeffs(nc) {
        TI np = 1;
        for (int k = 0; k < dim; ++k) np *= s[k];
        data.assign(d, d + np * nc);
    }
    const CP &englobing_convex_polyhedron() const { return img.englobing_convex_polyhedron(); }
    TF measure() const { return img.measure(); }

    static Pt lo(const ConvexPolyhedron2<Pc> &cp) {
        if (cp.nb_points() == 0 && cp.sphere_radius > 0) return cp.sphere_center - cp.sphere_radius;
        return cp.min_position();
    }
    static Pt hi(const ConvexPolyhedron2<Pc> &cp) {
        if (cp.nb_points() == 0 && cp.sphere_radius > 0) return cp.sphere_center + cp.sphere_radius;
        return cp.max_position();
    }
    static Pt lo(const ConvexPolyhedron3<Pc> &cp) { return cp.min_position(); }
    static Pt hi(const ConvexPolyhedron3<Pc> &cp) { return cp.max_position(); }

    template <class F>
    void for_each_intersection(CP &cp, const F &f) const {
        TI np = 1;
        for (int k = 0; k < dim; ++k) np *= sizes[k];
        if (np == 1) {
            SpaceFunctions::apply_poly(N<dim>(), data.data(), np, nb_coeffs, [&](const auto &sf) { return f(cp, sf); });
            return;
        }
        if (cp.nb_points() == 0 && !(cp.sphere_radius > 0)) return;  // void cell: nothing to integrate
        Pt ps;
        std::array<TI, dim> min_i, max_i;
        Pt min_pos = lo(cp), max_pos = hi(cp);
        for (int d = 0; d < dim; ++d) {
            TF mi = std::max(min_pos[d], min_pt[d]);
            TF ma = std::min(max_pos[d], max_pt[d]);
            min_i[d] = (mi - min_pt[d]) * sizes[d] / (max_pt[d] - min_pt[d]);
            max_i[d] = (ma - min_pt[d]) * sizes[d] / (max_pt[d] - min_pt[d]);
            min_i[d] = std::max(TI(1), min_i[d]) - 1;
            max_i[d] = std::min(sizes[d], max_i[d] + 2);
            ps[d] = (max_pt[d] - min_pt[d]) / sizes[d];
        }
        CP ccp;
        CrossProdOfRanges<TI, dim> cr(min_i, max_i);
        cr.for_each([&](auto p) {
            Pt pf;
            TI num_pix = 0, acc = 1;
            for (int d = 0; d < dim; ++d) {
                num_pix += acc * p[d];
                acc *= sizes[d];
                pf[d] = p[d];
            }
            ccp = {typename CP::Box{min_pt + ps * (pf + TF(0)), min_pt + ps * (pf + TF(1))}, typename Pc::CI(-1)};
            ccp.intersect_with(cp);
            SpaceFunctions::apply_poly(N<dim>(), data.data() + num_pix, acc, nb_coeffs, [&](const auto &sf) { f(ccp, sf); });
        });
    }
};

struct CtxBase {
    virtual ~CtxBase() {}
    std::vector<std::size_t> offsets, columns;
    std::vector<double> values, v_values;
    std::vector<std::int64_t> nb_offsets, nb_ids;
    double t_update = 0, t_integrals = 0, t_centroids = 0, t_der = 0;
};

double now() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

template <class Pc>
struct Ctx : CtxBase {
    static constexpr int dim = Pc::dim;
    using Grid = SpZGrid<Pc>;
    using Pt = typename Grid::Pt;
    using TF = double;
    using Assembly = ConvexPolyhedronAssembly<Pc>;
    using Image = FixedScaledImage<Pc>;

    Grid grid;
    Assembly assembly;
    std::unique_ptr<Image> image;
    std::vector<Pt> pos;
    std::vector<TF> w;
    bool ball_cut = false;

    explicit Ctx(std::size_t max_diracs_per_cell) : grid(max_diracs_per_cell) {}

    void set_diracs(std::int64_t n, const double *p, const double *ww) {
        pos.resize(n);
        w.assign(ww, ww + n);
        for (std::int64_t i = 0; i < n; ++i)
            for (int d = 0; d < dim; ++d) pos[i][d] = p[dim * i + d];
    }

    template <class F>
    void with_bounds_and_rf(const F &f) {
        if (image) {
            if (ball_cut) f(*image, FunctionEnum::InBallW05());
            else f(*image, FunctionEnum::Unit());
        } else {
            if (ball_cut) f(assembly, FunctionEnum::InBallW05());
            else f(assembly, FunctionEnum::Unit());
        }
    }

    void update() {
        double t0 = now();
        grid.update(pos.data(), w.data(), w.size());
        t_update = now() - t0;
    }

    void integrals(double *out) {
        double t0 = now();
        with_bounds_and_rf([&](auto &bounds, auto rf) {
            get_integrals(out, grid, bounds, pos.data(), w.data(), w.size(), rf);
        });
        t_integrals = now() - t0;
    }

    void centroids(double *out_c, double *out_m) {
        double t0 = now();
        with_bounds_and_rf([&](auto &bounds, auto rf) {
            get_centroids(grid, bounds, pos.data(), w.data(), w.size(), rf, [&](auto c, auto m, auto num) {
                for (int d = 0; d < dim; ++d) out_c[dim * num + d] = c[d];
                if (out_m) out_m[num] = m;
            });
        });
        t_centroids = now() - t0;
    }

    int der(int stop_if_void) {
        double t0 = now();
        int err = 0;
        with_bounds_and_rf([&](auto &bounds, auto rf) {
            err = get_der_integrals_wrt_weights(offsets, columns, values, v_values, grid, bounds, pos.data(), w.data(),
                                                w.size(), rf, bool(stop_if_void));
        });
        t_der = now() - t0;
        return err;
    }

    // get_der_centroids_and_integrals_wrt_weight_and_positions
    // (get_der_centroids_and_integrals_wrt_weight_and_positions.h:17-216), into
    // the der* members (offsets of (dim + 1) n rows)
    std::vector<std::size_t> dp_offsets, dp_columns;
    std::vector<double> dp_values, dp_v;
    int der_pos() {
        int err = 0;
        with_bounds_and_rf([&](auto &bounds, auto rf) {
            err = get_der_centroids_and_integrals_wrt_weight_and_positions(dp_offsets, dp_columns, dp_values, dp_v, grid,
                                                                           bounds, pos.data(), w.data(), w.size(), rf,
                                                                           false);
        });
        return err;
    }

    // get_image_integrals (get_image_integrals.h:16-78) and
    // get_image_of_cell_nums (get_image_of_cell_nums.h:13-80), 2D
    void image_integrals(const double *lo, const double *hi, const std::int64_t *nbp, double *out, bool nums,
                         std::int64_t *out_nums) {
        if constexpr (dim == 2) {
            Pt a, b;
            std::array<std::size_t, dim> s;
            for (int d = 0; d < dim; ++d) { a[d] = lo[d]; b[d] = hi[d]; s[d] = std::size_t(nbp[d]); }
            with_bounds_and_rf([&](auto &bounds, auto rf) {
                if (nums) {
                    std::vector<std::size_t> r(s[0] * s[1]);
                    get_image_of_cell_nums(r.data(), grid, bounds, pos.data(), w.data(), w.size(), rf, a, b, s);
                    for (std::size_t i = 0; i < r.size(); ++i) out_nums[i] = std::int64_t(r[i]);
                } else {
                    get_image_integrals(out, grid, bounds, pos.data(), w.data(), w.size(), rf, a, b, s);
                }
            });
        }
    }

    // cut ids of the final cell boundary (before any bounds intersection),
    // one list per Dirac: what the traversal hands to the callback.
    void neighbors() {
        std::size_t n = w.size();
        std::vector<std::vector<std::int64_t>> lists(n);
        with_bounds_and_rf([&](auto &bounds, auto rf) {
            grid.for_each_laguerre_cell(
                [&](auto &lc, std::size_t num, int) {
                    std::vector<std::int64_t> &l = lists[num];
                    collect(lc, l);
                },
                bounds.englobing_convex_polyhedron(), pos.data(), w.data(), n, false, bool(rf.need_ball_cut()));
        });
        nb_offsets.assign(n + 1, 0);
        nb_ids.clear();
        for (std::size_t i = 0; i < n; ++i) {
            nb_offsets[i] = nb_ids.size();
            nb_ids.insert(nb_ids.end(), lists[i].begin(), lists[i].end());
        }
        nb_offsets[n] = nb_ids.size();
    }

    static void collect(const ConvexPolyhedron2<Pc> &lc, std::vector<std::int64_t> &l) {
        for (std::size_t k = 0; k < lc.nb_points(); ++k)
            l.push_back(lc.arcs[k] ? -2 : std::int64_t(lc.cut_ids[k]));
    }
    static void collect(const ConvexPolyhedron3<Pc> &lc, std::vector<std::int64_t> &l) {
        lc.for_each_boundary_measure(SpaceFunctions::Constant<double>{1.0}, FunctionEnum::Unit(),
                                     [&](double, std::size_t id) { l.push_back(std::int64_t(id)); });
    }
};

template <class F>
auto dispatch(void *h, const F &f) {
    CtxBase *b = static_cast<CtxBase *>(h);
    if (auto *c2 = dynamic_cast<Ctx<Pc2> *>(b)) return f(*c2);
    return f(*dynamic_cast<Ctx<Pc3> *>(b));
}

}  // namespace

extern "C" {

void ref_init_threads(int nb_threads) { thread_pool.init(nb_threads); }
int ref_nb_threads() { return thread_pool.nb_threads(); }

void *ref_create(int dim, std::int64_t max_diracs_per_cell) {
    if (dim == 2) return static_cast<CtxBase *>(new Ctx<Pc2>(max_diracs_per_cell));
    if (dim == 3) return static_cast<CtxBase *>(new Ctx<Pc3>(max_diracs_per_cell));
    return nullptr;
}
void ref_destroy(void *h) { delete static_cast<CtxBase *>(h); }

void ref_set_diracs(void *h, std::int64_t n, const double *pos, const double *w) {
    dispatch(h, [&](auto &c) { c.set_diracs(n, pos, w); return 0; });
}
void ref_set_ball_cut(void *h, int on) {
    dispatch(h, [&](auto &c) { c.ball_cut = on != 0 && c.dim == 2; return 0; });
}

// ConvexPolyhedronAssembly::add_box (ConvexPolyhedronAssembly.tcc:46-50)
void ref_add_box(void *h, const double *p0, const double *p1, double coeff) {
    dispatch(h, [&](auto &c) {
        using Pt = typename std::decay_t<decltype(c)>::Pt;
        Pt a, b;
        for (int d = 0; d < c.dim; ++d) { a[d] = p0[d]; b[d] = p1[d]; }
        c.assembly.add_box(a, b, coeff);
        return 0;
    });
}
// ConvexPolyhedronAssembly::add_convex_polyhedron (ConvexPolyhedronAssembly.tcc:7-33)
void ref_add_convex_polyhedron(void *h, std::int64_t m, const double *pts, const double *nrm, double coeff) {
    dispatch(h, [&](auto &c) {
        using Pt = typename std::decay_t<decltype(c)>::Pt;
        std::vector<Pt> pv(m), nv(m);
        for (std::int64_t i = 0; i < m; ++i)
            for (int d = 0; d < c.dim; ++d) { pv[i][d] = pts[c.dim * i + d]; nv[i][d] = nrm[c.dim * i + d]; }
        c.assembly.add_convex_polyhedron(pv, nv, coeff);
        return 0;
    });
}
// ConvexPolyhedronAssembly::add_simplex (ConvexPolyhedronAssembly.tcc:36-43), 2D only here
void ref_add_simplex(void *h, const double *pts, double coeff) {
    dispatch(h, [&](auto &c) {
        if constexpr (std::decay_t<decltype(c)>::dim == 2) c.assembly.add_simplex(pts, coeff);
        return 0;
    });
}
void ref_normalize(void *h) { dispatch(h, [&](auto &c) { c.assembly.normalize(); return 0; }); }
double ref_domain_measure(void *h) {
    return dispatch(h, [&](auto &c) -> double { return c.image ? c.image->measure() : c.assembly.measure(); });
}

void ref_set_image(void *h, const double *min_pt, const double *max_pt, const double *data, const std::int64_t *sizes,
                   std::int64_t nb_coeffs) {
    dispatch(h, [&](auto &c) {
        using C = std::decay_t<decltype(c)>;
        using Pt = typename C::Pt;
        Pt a, b;
        std::array<std::size_t, C::dim> s;
        for (int d = 0; d < C::dim; ++d) { a[d] = min_pt[d]; b[d] = max_pt[d]; s[d] = sizes[d]; }
        c.image.reset(new typename C::Image(a, b, data, s, nb_coeffs));
        return 0;
    });
}

void ref_update(void *h) { dispatch(h, [&](auto &c) { c.update(); return 0; }); }
// SpZGrid::translations (2D)
void ref_set_translations(void *h, const double *t, std::int64_t count) {
    dispatch(h, [&](auto &c) {
        using Pt = typename std::decay_t<decltype(c)>::Pt;
        c.grid.translations.clear();
        for (std::int64_t k = 0; k < count; ++k) {
            Pt p;
            for (int d = 0; d < c.dim; ++d) p[d] = t[c.dim * k + d];
            c.grid.translations.push_back(p);
        }
        return 0;
    });
}
void ref_get_image_integrals(void *h, const double *lo, const double *hi, const std::int64_t *nbp, double *out) {
    dispatch(h, [&](auto &c) { c.image_integrals(lo, hi, nbp, out, false, nullptr); return 0; });
}
void ref_get_image_of_cell_nums(void *h, const double *lo, const double *hi, const std::int64_t *nbp,
                                std::int64_t *out) {
    dispatch(h, [&](auto &c) { c.image_integrals(lo, hi, nbp, nullptr, true, out); return 0; });
}
void ref_get_integrals(void *h, double *out) { dispatch(h, [&](auto &c) { c.integrals(out); return 0; }); }
void ref_get_centroids(void *h, double *out_c, double *out_m) {
    dispatch(h, [&](auto &c) { c.centroids(out_c, out_m); return 0; });
}
int ref_get_der_integrals_wrt_weights(void *h, int stop_if_void) {
    return dispatch(h, [&](auto &c) { return c.der(stop_if_void); });
}
std::int64_t ref_der_nnz(void *h) { return static_cast<CtxBase *>(h)->columns.size(); }
// position derivatives (2D): computes, returns nnz; then ref_der_pos_copy
std::int64_t ref_der_pos(void *h) {
    return dispatch(h, [&](auto &c) -> std::int64_t {
        if (c.der_pos()) return -1;
        return std::int64_t(c.dp_columns.size());
    });
}
void ref_der_pos_copy(void *h, std::int64_t *offsets, std::int64_t *columns, double *values, double *v) {
    dispatch(h, [&](auto &c) {
        for (std::size_t i = 0; i < c.dp_offsets.size(); ++i) offsets[i] = std::int64_t(c.dp_offsets[i]);
        for (std::size_t i = 0; i < c.dp_columns.size(); ++i) columns[i] = std::int64_t(c.dp_columns[i]);
        std::memcpy(values, c.dp_values.data(), c.dp_values.size() * sizeof(double));
        std::memcpy(v, c.dp_v.data(), c.dp_v.size() * sizeof(double));
        return 0;
    });
}
void ref_der_copy(void *h, std::int64_t *offsets, std::int64_t *columns, double *values, double *masses) {
    CtxBase *b = static_cast<CtxBase *>(h);
    for (std::size_t i = 0; i < b->offsets.size(); ++i) offsets[i] = b->offsets[i];
    for (std::size_t i = 0; i < b->columns.size(); ++i) columns[i] = b->columns[i];
    std::memcpy(values, b->values.data(), b->values.size() * sizeof(double));
    std::memcpy(masses, b->v_values.data(), b->v_values.size() * sizeof(double));
}
std::int64_t ref_neighbors(void *h) {
    dispatch(h, [&](auto &c) { c.neighbors(); return 0; });
    return static_cast<CtxBase *>(h)->nb_ids.size();
}
void ref_neighbors_copy(void *h, std::int64_t *offsets, std::int64_t *ids) {
    CtxBase *b = static_cast<CtxBase *>(h);
    std::memcpy(offsets, b->nb_offsets.data(), b->nb_offsets.size() * sizeof(std::int64_t));
    std::memcpy(ids, b->nb_ids.data(), b->nb_ids.size() * sizeof(std::int64_t));
}
void ref_timings(void *h, double *t4) {
    CtxBase *b = static_cast<CtxBase *>(h);
    t4[0] = b->t_update; t4[1] = b->t_integrals; t4[2] = b->t_centroids; t4[3] = b->t_der;
}

}  // extern "C"
