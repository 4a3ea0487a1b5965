// 2D Laguerre-cell kernels (sm_100a), FP64.
//
// One thread builds one cell.  Threads take Diracs in Morton (sorted) order so
// a warp works on 32 neighbouring cells and walks nearly the same tree nodes.
// The fast tier keeps the cell polygon in shared memory (SoA, one column per
// thread); cells that outgrow it are rebuilt by the big and huge tiers whose
// polygons live in global scratch (one column per thread, coalesced).  The
// traversal stack lives in local memory.
//
// Reference behaviour restated here:
//  * traversal, eviction test and bisector cuts: SpZGrid::for_each_laguerre_cell
//    (src/sdot/PowerDiagram/Visitors/SpZGrid.tcc:494-719, eviction :475-480,
//    bisector :506-522); the reference pops boxes best-first from a priority
//    queue keyed on the float distance to the box centre, here a depth-first
//    walk pushes children farthest-first so the nearest is visited first.
//  * disc clipping (InBallW05, ball_cut after all plane cuts): :633-634.
//  * integrals: ConvexPolyhedron2::integration(Constant,Unit)
//    (ConvexPolyhedron2.tcc:1791-1843), add_centroid_contrib (:1047-1074),
//    for_each_boundary_item (:437-478).
//  * Hessian row: get_der_integrals_wrt_weights (get_der_integrals_wrt_weights.h:43-88):
//    off-diagonal -1/2 * len_ij / |x_i - x_j|, diagonal the sum of those plus
//    1/2 * arc_len / sqrt(w_i).
//  * bounds: ConvexPolyhedronAssembly::for_each_intersection
//    (ConvexPolyhedronAssembly.tcc:132-142) and ScaledImage::for_each_intersection
//    (ScaledImage.tcc:98-149).  A piece (cell intersected with an item or a
//    pixel) is produced by clipping the cell by the item/pixel half-planes,
//    which is the same convex set the reference gets by clipping the item by
//    the cell's lines.
#include "cell2d.cuh"
#include "geom2d.cuh"

namespace sdot {

// Counting builds (-DSDOT_COUNT) add up the work of the fast tier's walks,
// the terms of the per-cell operation count: [0] cut attempts, [1] vertices
// classified at them, [2] node tests, [3] vertices tested at them, [4]
// effective cuts, [5] final vertices, [6] cells built.  Release builds
// compile the counting away.
#ifdef SDOT_COUNT
static __device__ unsigned long long sdot_work[8];
#define SDOT_WORK_ADD(k, v) atomicAdd(&sdot_work[k], (unsigned long long)(v))
#else
#define SDOT_WORK_ADD(k, v) ((void)0)
#endif

namespace {

constexpr int T2D_MAX = 128;  // largest block of the fast kernels (their block size is tuned, see launch_all)
constexpr int STACK = 64;   // traversal stack (depth <= 17 levels, <= 3 pending siblings each)
constexpr int WTIER_WARPS = 148 * 4;  // warps of the warp-per-cell tier (4 per SM; 8 or 16 measured no faster)

// Records the first failed consistency guard and flags the error word; the
// caller then skips the access.  Guards cover every index that comes from
// data (tree nodes, leaf ranges, item offsets), so a corrupt input gives an
// error status instead of a fault.
SDOT_KFN void guard_fail(const Cell2DArgs &A, int code, long long s, long long value) {
#ifdef __CUDA_ARCH__
    const bool first = A.guard && atomicCAS(&A.guard[0], 0, code) == 0;
#else
    const bool first = A.guard && A.guard[0] == 0;
    if (first) A.guard[0] = code;
#endif
    if (first) {
        A.guard[1] = int(s);
        A.guard[2] = int(value);
    }
    flag_error(A.err, DE_GUARD);
}

// Destination of one row (or id list): element k at col[k * stride]
// (col == nullptr: the output is not wanted, only counted).
struct Out {
    int *col;
    double *val;
    long long stride;
    int cap;
    int cnt = 0;
    SDOT_HDI Out(int *c, double *v, long long st, int cp) : col(c), val(v), stride(st), cap(cp) {}
    SDOT_HDI void emit(int j, double v) {
        if (col && cnt < cap) {
            col[cnt * stride] = j;
            if (val) val[cnt * stride] = v;
        }
        ++cnt;
    }
    SDOT_HDI bool ok() const { return !col || cnt <= cap; }
};

// Integrates a streamed polygon (one piece at a time) and collects the
// boundary measures for the Hessian row.  P: the cell's polygon view (its
// ids name the neighbours).  POLY: the density of a piece is the quadratic
// c0 + c1 x + c2 y + c3 x^2 + c4 x y + c5 y^2 (absolute coordinates) of a
// piecewise-quadratic image (ScaledImage with nb_coeffs = 6), integrated
// exactly: the edge-midpoint rule on each fan triangle for the mass (exact
// for quadratics), the 7-point rule (vertices 1/20, edge midpoints 2/15,
// centroid 9/20 of the area; exact for cubics) for the first moments, and
// Simpson's rule along each edge for the boundary measures (exact for
// quadratics).  The reference evaluates the same integrals from expanded
// closed forms (ConvexPolyhedron2.tcc:2181-2225 integration, :980-1044
// add_centroid_contrib, :180-214 for_each_boundary_item).
template <bool DIRECT, class P = PolyView<double>, bool POLY = false>
struct Sink {
    const P &cell;
    const double *pos;
    double c0x, c0y, sqw0;
    double cx, cy, r;
    double coeff = 1.0;
    // piece state
    bool has_first = false;
    double fx = 0, fy = 0, px = 0, py = 0;
    int ft = 0, pt = 0, cnt = 0;
    double tr2 = 0, arcs = 0, pm = 0, pcx = 0, pcy = 0;
    // cell totals
    double mass = 0, mass_c = 0, momx = 0, momy = 0, der0 = 0;
    // rows: DIRECT emits one item per line edge; otherwise measures are
    // summed per cell edge in acc (negative = edge not seen yet)
    double *acc;
    int acc_st;
    Out &row;
    long long n_diracs = 1LL << 40;
    const double *trans = nullptr;  // periodic domains: translation k of id j + (k + 1) n

    SDOT_HDI Sink(const P &c, const double *p, double x0, double y0, double sw, double r_, double *a, int ast,
                  Out &ro)
        : cell(c), pos(p), c0x(x0), c0y(y0), sqw0(sw), cx(x0), cy(y0), r(r_), acc(a), acc_st(ast), row(ro) {}

    double q[6] = {0, 0, 0, 0, 0, 0};  // POLY: the piece's density coefficients

    SDOT_HDI void begin_piece(double c) {
        coeff = c;
        has_first = false;
        cnt = 0;
        tr2 = arcs = pm = pcx = pcy = 0;
    }
    // POLY: the coefficients of pixel p, plane k at c[p + k * plane]
    SDOT_HDI void begin_piece_poly(const double *c, long long plane) {
        for (int k = 0; k < 6; ++k) q[k] = c[k * plane];
        begin_piece(1.0);
    }
    SDOT_HDI double f(double x, double y) const {
        return q[0] + q[1] * x + q[2] * y + q[3] * x * x + q[4] * x * y + q[5] * y * y;
    }
    SDOT_HDI void line(int t, double len) {
        if (t < 0) return;
        const int id = cell.I(t);
        if (id < 0) return;
        const double m = coeff * len;
        if (DIRECT) {
            // the neighbour, or the image of Dirac j under translation k for
            // an id j + (k + 1) n (get_der_integrals_wrt_weights.h:61-62)
            int j = id;
            double qx, qy;
            if (id >= n_diracs) {
                const int k = int(id / n_diracs) - 1;
                j = int(id % n_diracs);
                qx = pos[2 * j] + trans[2 * k];
                qy = pos[2 * j + 1] + trans[2 * k + 1];
            } else {
                qx = pos[2 * SDOT_CHECK_IDX(id, n_diracs, 3)];
                qy = pos[2 * id + 1];
            }
            const double dx = c0x - qx, dy = c0y - qy;
            const double dist = sqrt(dx * dx + dy * dy);
            if (dist != 0) {
                const double b = 0.5 * m / dist;
                row.emit(j, -b);
                der0 += b;
            }
        } else {
            double &a = acc[SDOT_CHECK_IDX(t, cell.cap, 2) * acc_st];
            a = a < 0 ? m : a + m;
        }
    }
    SDOT_HDI void edge(double ax, double ay, int t, double bx, double by) {
        if (t == ID_ARC) {
            arcs += arc_area(ax, ay, bx, by, cx, cy, r);
            centroid_arc(pcx, pcy, pm, ax, ay, bx, by, cx, cy, r, coeff);
            double a0;
            const double a1 = arc_angles(ax, ay, bx, by, cx, cy, a0);
            der0 += 0.5 * (coeff * (a1 - a0) * r) / sqw0;
        } else {
            const double dx = bx - ax, dy = by - ay;
            const double len = sqrt(dx * dx + dy * dy);
            if (POLY)  // Simpson along the edge; line() multiplies by coeff = 1
                line(t, len * (1.0 / 6.0) * (f(ax, ay) + 4.0 * f(0.5 * (ax + bx), 0.5 * (ay + by)) + f(bx, by)));
            else
                line(t, len);
        }
    }
    SDOT_HDI void push(double x, double y, int tag) {
        if (!has_first) {
            has_first = true;
            fx = x; fy = y; ft = tag;
        } else {
            edge(px, py, pt, x, y);
        }
        if (++cnt >= 3) {
            const double t2 = fx * (py - y) + px * (y - fy) + x * (fy - py);
            tr2 += t2;
            if (POLY) {
                const double a = 0.5 * t2;
                const double m1x = 0.5 * (fx + px), m1y = 0.5 * (fy + py), m2x = 0.5 * (px + x), m2y = 0.5 * (py + y);
                const double m3x = 0.5 * (x + fx), m3y = 0.5 * (y + fy);
                const double gx = (1.0 / 3.0) * (fx + px + x), gy = (1.0 / 3.0) * (fy + py + y);
                const double f1 = f(m1x, m1y), f2 = f(m2x, m2y), f3 = f(m3x, m3y);
                const double fa = f(fx, fy), fb = f(px, py), fc = f(x, y), fg = f(gx, gy);
                pm += a * (1.0 / 3.0) * (f1 + f2 + f3);
                pcx += a * ((1.0 / 20.0) * (fx * fa + px * fb + x * fc) +
                            (2.0 / 15.0) * (m1x * f1 + m2x * f2 + m3x * f3) + (9.0 / 20.0) * gx * fg);
                pcy += a * ((1.0 / 20.0) * (fy * fa + py * fb + y * fc) +
                            (2.0 / 15.0) * (m1y * f1 + m2y * f2 + m3y * f3) + (9.0 / 20.0) * gy * fg);
            } else {
                const double lea = 0.5 * t2 * coeff;
                const double f = (1.0 / 3.0) * lea;
                pcx += f * (fx + px + x);
                pcy += f * (fy + py + y);
                pm += lea;
            }
        }
        px = x; py = y; pt = tag;
    }
    SDOT_HDI void finish() {
        if (has_first) edge(px, py, pt, fx, fy);
    }
    // radius: the disc radius after clipping (> 0 keeps a vertex-free piece
    // as the full disc), or -1 when there is no disc.
    SDOT_HDI void end_piece(double radius) {
        if (cnt == 0) {
            if (radius > 0) {
                const double lea = kPi * (radius * radius) * coeff;
                mass += lea;
                mass_c += lea;
                momx += lea * cx;
                momy += lea * cy;
                der0 += 0.5 * (coeff * 2 * kPi * radius) / sqw0;
            }
            return;
        }
        mass += POLY ? pm : coeff * (tr2 * 0.5 + arcs);
        mass_c += pm;
        momx += pcx;
        momy += pcy;
    }
};

// Area of a streamed (clipped) polygon, segments of the clipping disc
// included (fan from the first vertex plus the arc segments, as Sink).
struct AreaSink {
    double cx, cy, r;
    bool has_first = false;
    double fx = 0, fy = 0, px = 0, py = 0;
    int pt = 0, cnt = 0;
    double tr2 = 0, arcs = 0;
    SDOT_HDI AreaSink(double x, double y, double rr) : cx(x), cy(y), r(rr) {}
    SDOT_HDI void edge(double ax, double ay, int t, double bx, double by) {
        if (t == ID_ARC) arcs += arc_area(ax, ay, bx, by, cx, cy, r);
    }
    SDOT_HDI void push(double x, double y, int tag) {
        if (!has_first) {
            has_first = true;
            fx = x;
            fy = y;
        } else {
            edge(px, py, pt, x, y);
        }
        if (++cnt >= 3) tr2 += fx * (py - y) + px * (y - fy) + x * (fy - py);
        px = x;
        py = y;
        pt = tag;
    }
    SDOT_HDI void finish() {
        if (has_first) edge(px, py, pt, fx, fy);
    }
    // radius: the disc radius after clipping (> 0 keeps a vertex-free piece
    // as the full disc), or -1 when there is no disc
    SDOT_HDI double area(double radius) const {
        if (cnt == 0) return radius > 0 ? kPi * radius * radius : 0.0;
        return 0.5 * tr2 + arcs;
    }
};

// Integrates the cell of sorted Dirac s (its polygon before disc clipping,
// n vertices) over the pixels of the raster that its bounding box meets:
// get_image_integrals / get_image_of_cell_nums
// (get_image_integrals.h:16-78, get_image_of_cell_nums.h:13-80) clip each
// pixel box by the cell and integrate; here the cell is clipped by the pixel's
// four lines (and the disc), the same convex set.
template <bool BALL, class P>
SDOT_KFN void raster_cell(const Cell2DArgs &A, long long s, const P &cell, int n, double c0x, double c0y,
                          double r) {
    if (n <= 0) return;
    double xmin = cell.X(0), xmax = xmin, ymin = cell.Y(0), ymax = ymin;
    for (int k = 1; k < n; ++k) {
        xmin = fmin(xmin, cell.X(k)); xmax = fmax(xmax, cell.X(k));
        ymin = fmin(ymin, cell.Y(k)); ymax = fmax(ymax, cell.Y(k));
    }
    if (BALL) {
        xmin = fmax(xmin, c0x - r); xmax = fmin(xmax, c0x + r);
        ymin = fmax(ymin, c0y - r); ymax = fmin(ymax, c0y + r);
    }
    const double psx = (A.ras_hi[0] - A.ras_lo[0]) / A.ras_nx, psy = (A.ras_hi[1] - A.ras_lo[1]) / A.ras_ny;
    const double fx0 = floor((xmin - A.ras_lo[0]) / psx), fx1 = floor((xmax - A.ras_lo[0]) / psx);
    const double fy0 = floor((ymin - A.ras_lo[1]) / psy), fy1 = floor((ymax - A.ras_lo[1]) / psy);
    if (!(fx1 >= 0 && fy1 >= 0 && fx0 < A.ras_nx && fy0 < A.ras_ny)) return;  // outside the raster (or NaN)
    const int ix0 = int(fmax(fx0, 0.0)), ix1 = int(fmin(fx1, double(A.ras_nx - 1)));
    const int iy0 = int(fmax(fy0, 0.0)), iy1 = int(fmin(fy1, double(A.ras_ny - 1)));
    const long long orig = A.perm ? A.perm[s] : s;
    for (int iy = iy0; iy <= iy1; ++iy) {
        const double y0 = A.ras_lo[1] + psy * double(iy), y1 = A.ras_lo[1] + psy * double(iy + 1);
        for (int ix = ix0; ix <= ix1; ++ix) {
            const double x0 = A.ras_lo[0] + psx * double(ix), x1 = A.ras_lo[0] + psx * double(ix + 1);
            AreaSink as(c0x, c0y, r);
            double m;
            if (BALL) {
                DiscClip<AreaSink> dc(as, c0x, c0y, r);
                AxisClip<DiscClip<AreaSink>> c4(dc, 1, y1, -1.0, PID_OWN);
                AxisClip<AxisClip<DiscClip<AreaSink>>> c3(c4, 1, y0, 1.0, PID_OWN);
                AxisClip<AxisClip<AxisClip<DiscClip<AreaSink>>>> c2(c3, 0, x1, -1.0, PID_OWN);
                AxisClip<AxisClip<AxisClip<AxisClip<DiscClip<AreaSink>>>>> c1(c2, 0, x0, 1.0, PID_OWN);
                stream_cell(cell, n, c1);
                m = A.coeff * as.area(dc.result_radius());
            } else {
                AxisClip<AreaSink> c4(as, 1, y1, -1.0, PID_OWN);
                AxisClip<AxisClip<AreaSink>> c3(c4, 1, y0, 1.0, PID_OWN);
                AxisClip<AxisClip<AxisClip<AreaSink>>> c2(c3, 0, x1, -1.0, PID_OWN);
                AxisClip<AxisClip<AxisClip<AxisClip<AreaSink>>>> c1(c2, 0, x0, 1.0, PID_OWN);
                stream_cell(cell, n, c1);
                m = A.coeff * as.area(-1.0);
            }
            if (m == 0) continue;
            const long long pix = (long long)iy * A.ras_nx + ix;
#ifdef __CUDA_ARCH__
            if (A.ras) {
                atomicAdd(&A.ras[3 * pix], m * c0x);
                atomicAdd(&A.ras[3 * pix + 1], m * c0y);
                atomicAdd(&A.ras[3 * pix + 2], m);
            }
            if (A.ras_nums) atomicMax(&A.ras_nums[pix], orig);
#else
            if (A.ras) {
                A.ras[3 * pix] += m * c0x;
                A.ras[3 * pix + 1] += m * c0y;
                A.ras[3 * pix + 2] += m;
            }
            if (A.ras_nums && A.ras_nums[pix] < orig) A.ras_nums[pix] = orig;
#endif
        }
    }
}

// Records the ids of the streamed (disc-clipped) cell boundary.
template <class P = PolyView<double>>
struct NbSink {
    const P &cell;
    Out &out;
    SDOT_HDI NbSink(const P &c, Out &o) : cell(c), out(o) {}
    SDOT_HDI void push(double, double, int tag) { out.emit(tag == ID_ARC ? ID_ARC : cell.I(tag), 0.0); }
    SDOT_HDI void finish() {}
};

// Streams a polygon; each vertex carries the index of the cell edge leaving
// it: for the cell itself that is the vertex index, for a piece (a clipped
// copy of the cell) it is the tag stored in its id slot.
template <class Stage, class P>
SDOT_HDI void stream_cell(const P &cell, int n, Stage &st) {
    for (int k = 0; k < n; ++k) st.push(cell.X(k), cell.Y(k), k);
    st.finish();
}

// The children [first, first + nch) of a box (2 <= nch <= 4) in ch[0 ..
// nch), farthest first by the float squared distance from c0 to their box
// centres (the key of the reference's queue), the box shifted by (tx, ty)
// when PER.  A fixed network of five exchanges over four slots (missing
// children keyed -1, after every real key) keeps the arrays in registers.
template <bool PER>
SDOT_HDI void order_children(const Cell2DArgs &A, int first, int nch, double c0x, double c0y, double tx, double ty,
                             int ch[4]) {
    float key[4] = {-1.f, -1.f, -1.f, -1.f};
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        ch[c] = first + c;
        if (c < nch) {
            const TreeNode<2> &cn = A.nodes[SDOT_CHECK_IDX(first + c, A.max_nodes, 5)];
            const double cx = 0.5 * (cn.lo[0] + cn.hi[0]), cy = 0.5 * (cn.lo[1] + cn.hi[1]);
            const double mx = c0x - (PER ? cx + tx : cx);
            const double my = c0y - (PER ? cy + ty : cy);
            key[c] = float(mx * mx + my * my);
        }
    }
    auto cx = [&](int a, int b) {
        if (key[a] < key[b]) {
            const float tk = key[a];
            key[a] = key[b];
            key[b] = tk;
            const int tc = ch[a];
            ch[a] = ch[b];
            ch[b] = tc;
        }
    };
    cx(0, 1);
    cx(2, 3);
    cx(0, 2);
    cx(1, 3);
    cx(1, 2);
}

// Builds the Laguerre cell of sorted Dirac s (before any disc clipping) as a
// machine of uniform steps, so that the 32 cells of a warp advance together.
// The walk is SpZGrid::for_each_laguerre_cell's (SpZGrid.tcc:494-719): boxes
// popped nearest-first (children pushed farthest-first, keyed on the float
// squared distance from c0 to the box centre as the reference's queue),
// skipped when the eviction test holds for every vertex (SpZGrid.tcc:475-480),
// a leaf's Diracs cut in index order (bisector SpZGrid.tcc:506-522).
// Every step -- a node test or one cut -- is the same pass over the vertices:
// a cut classifies each vertex by its side of the bisector, a node test asks
// whether some vertex fails the eviction test; both quantities are computed
// for every vertex and the step's one is kept, so lanes on different kinds of
// steps run the same instructions.  Only the application of an effective cut
// and the handling of a needed node branch.
// Returns the vertex count, -1 on capacity (or stack / visit cap) overflow,
// -2 on a failed guard.
// PER (periodic domains): after the tree, the walk visits it again once per
// translation t, as the tree of the Diracs x_j + t (SpZGrid.tcc:558-561:
// every translation's root enters the front; boxes and Diracs are shifted by
// t, :396-397 and :608-611); a cut by the image of Dirac j under translation
// k carries the id j + (k + 1) n, and the Dirac's own images cut it too.
template <bool PER = false>
SDOT_KFN int build_cell(const Cell2DArgs &A, long long s, const PolyView<double> &cell, int cap, double c0x, double c0y,
                        double w0) {
    int n = A.start_n;
    for (int k = 0; k < n; ++k) {
        cell.X(k) = A.start_xy[2 * k];
        cell.Y(k) = A.start_xy[2 * k + 1];
        cell.I(k) = domain_id(k);
    }
    // The walk's memory reads are issued a step before their use, so that
    // their latency overlaps the vertex pass of the step before: the node
    // popped next is kept in a register (the stack holds the others), and the
    // position and weight of the next Dirac of a leaf are loaded while the
    // current one cuts.
    int stack[STACK];
    int sp = 0;                 // stack entries below `top`
    int top = 0;                // the node the next node step pops
    bool has_top = true;
    int j = 0, je = 0;          // Diracs of the current leaf still to cut by
    double cjx = 0, cjy = 0, cjw = 0;  // Dirac j
    int visits = 0;
    int sym = -1;               // PER: the translation of the current walk (-1: none)
    double tx = 0, ty = 0;      // and its vector
    auto skip_self = [&](int k) { return (!PER || sym < 0) && k == s ? k + 1 : k; };
    // shifted by the current translation (PER only: adding a zero would not
    // be free, it turns -0 into +0)
    auto tr = [&](double v, double t) { return PER ? v + t : v; };
    while (true) {
        // ---- the step: one cut (j < je) or one node test
        if (PER && j >= je && !has_top && sym + 1 < A.ntrans) {
            // the next translation's walk starts from the root again
            ++sym;
            tx = A.trans[2 * sym];
            ty = A.trans[2 * sym + 1];
            top = 0;
            has_top = true;
        }
        const bool is_cut = j < je;
        double ox = 0, oy = 0, nx = 0, ny = 0;
        double lo0 = 0, lo1 = 0, hi0 = 0, hi1 = 0, maxw = 0;
        int node = -1, nd_a = 0, nd_b = 0;
        int jn = 0;
        double njx = 0, njy = 0, njw = 0;
        if (is_cut) {
            bisector(c0x, c0y, w0, cjx, cjy, cjw, ox, oy, nx, ny);
            jn = skip_self(j + 1);
            if (jn < je) {
                (void)SDOT_CHECK_IDX(jn, A.n, 6);
                njx = tr(A.pos[2 * jn], tx);
                njy = tr(A.pos[2 * jn + 1], ty);
                njw = A.w[jn];
            }
        } else {
            if (!has_top) break;
            if (++visits > (PER ? (A.ntrans + 1) * A.max_nodes : A.max_nodes)) {  // each tree walk visits a node once
                flag_error(A.err, DE_ITER);
                return -1;
            }
            node = top;
            if (sp > 0)
                top = stack[--sp];
            else
                has_top = false;
            const TreeNode<2> &nd = A.nodes[SDOT_CHECK_IDX(node, A.max_nodes, 4)];
            lo0 = tr(nd.lo[0], tx);
            lo1 = tr(nd.lo[1], ty);
            hi0 = tr(nd.hi[0], tx);
            hi1 = tr(nd.hi[1], ty);
            maxw = nd.maxw;
            nd_a = nd.a;
            nd_b = nd.b;
        }
        // ---- the pass over the vertices: a cut classifies each vertex by
        // its side of the bisector (bit k: vertex k outside); a node test
        // stops at the first vertex that fails the eviction test, as the
        // reference's all_pos does (mask 1: the box is needed)
        unsigned mask = 0;
        int tested = n;
        if (is_cut) {
            for (int k = 0; k < n; ++k) {
                const double d = (ox - cell.X(k)) * nx + (oy - cell.Y(k)) * ny;
                mask |= unsigned(d < 0.0) << k;
            }
        } else {
            for (int k = 0; k < n; ++k) {
                const double px = cell.X(k), py = cell.Y(k);
                const double qx = fmin(hi0, fmax(lo0, px)), qy = fmin(hi1, fmax(lo1, py));
                const double lhs = (c0x - px) * (c0x - px) + (c0y - py) * (c0y - py) - w0;
                const double rhs = (qx - px) * (qx - px) + (qy - py) * (qy - py) - maxw;
                if (!(lhs <= rhs)) {  // this vertex fails: the box is needed
                    mask = 1u;
                    tested = k + 1;
                    break;
                }
            }
        }
        (void)tested;
        const CutFacts f = cut_facts(mask, n);
        SDOT_WORK_ADD(is_cut ? 0 : 2, 1);
        SDOT_WORK_ADD(is_cut ? 1 : 3, tested);
        if (is_cut) {
            if (f.nb_out) {
                SDOT_WORK_ADD(4, 1);
                n = plane_cut_apply(cell, n, cap, ox, oy, nx, ny, PER ? j + (sym + 1) * int(A.n) : j, f);
                if (n <= 0) return n;
            }
            j = jn;
            cjx = njx;
            cjy = njy;
            cjw = njw;
            continue;
        }
        if (f.nb_out == 0) continue;  // every vertex passes: the box is evicted
        if (nd_b < 0) {
            const int first = nd_a, nch = -nd_b;
            if (nch < 2 || nch > 4 || first < 1 || first + nch > A.max_nodes) {
                guard_fail(A, 1, s, node);
                return -2;
            }
            if (sp + nch > STACK) {
                flag_error(A.err, DE_STACK);
                return -1;
            }
            int ch[4];
            order_children<PER>(A, first, nch, c0x, c0y, tx, ty, ch);
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                if (c < nch) {
                    if (has_top) stack[sp++] = top;
                    top = ch[c];
                    has_top = true;
                }
            }
        } else {
            if (nd_a < 0 || nd_b > A.n) {
                guard_fail(A, 2, s, node);
                return -2;
            }
            j = skip_self(nd_a);
            je = nd_b;
            if (j < je) {
                cjx = tr(A.pos[2 * j], tx);
                cjy = tr(A.pos[2 * j + 1], ty);
                cjw = A.w[j];
            }
        }
    }
    return n;
}

// ---------------------------------------------------------------- mixed FP32
// FP32 build of the cell of Dirac s for the mixed-precision path, in
// coordinates relative to c0 (vertex u = p - c0), so that the float error is
// relative to the size of the cell rather than of the domain.  Same walk and
// same steps as build_cell; the decisions are made safe this way:
//  * a box is evicted only when every vertex passes the eviction test by more
//    than the float rounding of its two sides (a wrong eviction could drop a
//    neighbour; an extra visit only costs time);
//  * a cut that classifies some vertex within the float rounding of the
//    bisector stops the build with -3: the caller rebuilds the cell in FP64.
// The polygon's edge ids then give the topology that the FP64 re-clip
// (ReclipView) turns into exact vertices.  Returns like build_cell, or -3.
constexpr float F32_MARGIN = 16.0f * 5.96e-8f;  // 16 float ulps, relative

SDOT_KFN int build_cell_f32(const Cell2DArgs &A, long long s, const PolyView<float> &cell, int cap, double c0x,
                            double c0y, double w0, bool local) {
    const float w0f = float(w0);
    int n = 0;
    float span = 0;  // size of the starting polygon: the scale of the vertices' rounding
    if (local) {
        // Start from a local square of half-size R around c0 cut by the
        // domain's edges, not from the domain itself: float vertices
        // interpolated along domain-sized edges would carry errors at the
        // domain's scale.  R is 3 times the farthest of the 12 Morton-order
        // neighbours.  The square is exact for the cell when none of its
        // edges survives (the eviction tests on the truncated polygon are
        // then valid for the whole cell); otherwise the cell is rebuilt in
        // FP64, or, when it only emptied within the square, walked again from
        // the whole domain (-4).
        double r2 = 0;
        for (long long q = s - 6; q <= s + 6; ++q) {
            if (q == s || q < 0 || q >= A.n) continue;
            const double dx = A.pos[2 * q] - c0x, dy = A.pos[2 * q + 1] - c0y;
            r2 = fmax(r2, dx * dx + dy * dy);
        }
        const float R = float(3.0 * sqrt(r2));
        if (!(R > 0)) return -3;
        span = 2 * R;
        n = 4;
        cell.X(0) = -R; cell.Y(0) = -R; cell.I(0) = ID_LOCAL;
        cell.X(1) = R;  cell.Y(1) = -R; cell.I(1) = ID_LOCAL;
        cell.X(2) = R;  cell.Y(2) = R;  cell.I(2) = ID_LOCAL;
        cell.X(3) = -R; cell.Y(3) = R;  cell.I(3) = ID_LOCAL;
        for (int e = 0; e < A.start_n && n > 0; ++e) {
            const int e1 = e + 1 < A.start_n ? e + 1 : 0;
            const double p0x = A.start_xy[2 * e] - c0x, p0y = A.start_xy[2 * e + 1] - c0y;
            const double dx = A.start_xy[2 * e1] - A.start_xy[2 * e];
            const double dy = A.start_xy[2 * e1 + 1] - A.start_xy[2 * e + 1];
            n = plane_cut(cell, n, cap, float(p0x), float(p0y), float(dy), float(-dx), domain_id(e));
        }
        if (n <= 0) return -4;  // the square misses the domain
    } else {
        // the whole domain: used to decide cells that emptied within the
        // square; a non-empty result goes to FP64
        n = A.start_n;
        for (int k = 0; k < n; ++k) {
            cell.X(k) = float(A.start_xy[2 * k] - c0x);
            cell.Y(k) = float(A.start_xy[2 * k + 1] - c0y);
            cell.I(k) = domain_id(k);
            span = fmaxf(span, fabsf(cell.X(k)) + fabsf(cell.Y(k)));
        }
        span *= 2;
    }
    auto has_local = [&]() {
        for (int k = 0; k < n; ++k)
            if (cell.I(k) == ID_LOCAL) return true;
        return false;
    };
    int stack[STACK];
    int sp = 0;
    stack[sp++] = 0;
    int j = 0, je = 0;
    int visits = 0;
    while (true) {
        const bool is_cut = j < je;
        float ox = 0, oy = 0, nx = 0, ny = 0;
        float lo0 = 0, lo1 = 0, hi0 = 0, hi1 = 0, maxw = 0;
        int node = -1, nd_a = 0, nd_b = 0;
        if (is_cut) {
            if (j == s) {
                ++j;
                continue;
            }
            (void)SDOT_CHECK_IDX(j, A.n, 6);
            const double vx = A.pos[2 * j] - c0x, vy = A.pos[2 * j + 1] - c0y;
            const double x = 0.5 + 0.5 * (w0 - A.w[j]) / (vx * vx + vy * vy);
            nx = float(vx);
            ny = float(vy);
            ox = float(x * vx);
            oy = float(x * vy);
        } else {
            if (sp == 0) break;
            if (++visits > A.max_nodes) {
                flag_error(A.err, DE_ITER);
                return -1;
            }
            node = stack[--sp];
            const TreeNode<2> &nd = A.nodes[SDOT_CHECK_IDX(node, A.max_nodes, 4)];
            lo0 = float(nd.lo[0] - c0x);
            lo1 = float(nd.lo[1] - c0y);
            hi0 = float(nd.hi[0] - c0x);
            hi1 = float(nd.hi[1] - c0y);
            maxw = float(nd.maxw);
            nd_a = nd.a;
            nd_b = nd.b;
        }
        // a cut classifies every vertex (and flags one too close to call);
        // a node test stops at the first vertex that fails the eviction
        // test by more than its rounding margin (mask 1: the box is needed)
        unsigned mask = 0;
        bool near = false;
        if (is_cut) {
            for (int k = 0; k < n; ++k) {
                const float px = cell.X(k), py = cell.Y(k);
                const float ex = ox - px, ey = oy - py;
                const float d = ex * nx + ey * ny;
                // rounding of d: the products, the bisector's origin, and the
                // vertex, whose error scales with the edges it was cut from
                near |= fabsf(d) <= F32_MARGIN * (fabsf(ex * nx) + fabsf(ey * ny) +
                                                  (fabsf(ox) + fabsf(px) + span) * fabsf(nx) +
                                                  (fabsf(oy) + fabsf(py) + span) * fabsf(ny));
                mask |= unsigned(d < 0.0f) << k;
            }
        } else {
            for (int k = 0; k < n; ++k) {
                const float px = cell.X(k), py = cell.Y(k);
                const float qx = fminf(hi0, fmaxf(lo0, px)) - px, qy = fminf(hi1, fmaxf(lo1, py)) - py;
                const float uu = px * px + py * py, qq = qx * qx + qy * qy;
                const float lhs = uu - w0f, rhs = qq - maxw;
                const float emargin = F32_MARGIN * (uu + fabsf(w0f) + qq + fabsf(maxw));
                if (!(lhs <= rhs - emargin)) {
                    mask = 1u;
                    break;
                }
            }
        }
        if (near) return -3;
        const CutFacts f = cut_facts(mask, n);
        if (is_cut) {
            if (f.nb_out) {
                if (f.nb_out == n && has_local()) return -4;  // empty within the square only
                n = plane_cut_apply(cell, n, cap, ox, oy, nx, ny, j, f);
                if (n <= 0) return n;
            }
            ++j;
            continue;
        }
        if (f.nb_out == 0) continue;
        if (nd_b < 0) {
            const int first = nd_a, nch = -nd_b;
            if (nch < 2 || nch > 4 || first < 1 || first + nch > A.max_nodes) {
                guard_fail(A, 1, s, node);
                return -2;
            }
            if (sp + nch > STACK) {
                flag_error(A.err, DE_STACK);
                return -1;
            }
            int ch[4];
            order_children<false>(A, first, nch, c0x, c0y, 0.0, 0.0, ch);
#pragma unroll
            for (int c = 0; c < 4; ++c)
                if (c < nch) stack[sp++] = ch[c];
        } else {
            if (nd_a < 0 || nd_b > A.n) {
                guard_fail(A, 2, s, node);
                return -2;
            }
            j = nd_a;
            je = nd_b;
        }
    }
    return has_local() ? -3 : n;
}

// The FP64 polygon of a cell whose topology came from the FP32 build: vertex
// k is the intersection of the lines of edges k - 1 and k (a weighted
// bisector, or an edge of the starting polygon), solved in FP64 in
// coordinates relative to c0 and shifted back.  X, Y, I as PolyView's.
struct ReclipView {
    const Cell2DArgs &A;
    PolyView<float> poly;
    int n;
    double c0x, c0y, w0;
    int cap = CAP_FAST_2D;  // vertex slots (bound of the debug checks)
    mutable int ck = -1;
    mutable double vx = 0, vy = 0;

    SDOT_HDI int I(int k) const { return poly.I(k); }
    // line a . u = b of the edge with this id (u relative to c0)
    SDOT_HDI void line(int id, double &ax, double &ay, double &b) const {
        if (id >= 0) {
            const double dx = A.pos[2 * id] - c0x, dy = A.pos[2 * id + 1] - c0y;
            ax = dx;
            ay = dy;
            b = 0.5 * (dx * dx + dy * dy) + 0.5 * (w0 - A.w[id]);
        } else {
            const int e = domain_edge(id), e1 = e + 1 < A.start_n ? e + 1 : 0;
            const double p0x = A.start_xy[2 * e] - c0x, p0y = A.start_xy[2 * e + 1] - c0y;
            const double p1x = A.start_xy[2 * e1] - c0x, p1y = A.start_xy[2 * e1 + 1] - c0y;
            ax = p0y - p1y;
            ay = p1x - p0x;
            b = ax * p0x + ay * p0y;
        }
    }
    // intersection of edges k - 1 and k; returns |sin| of their angle
    SDOT_HDI double solve(int k, double &ux, double &uy) const {
        double a1x, a1y, b1, a2x, a2y, b2;
        line(I(k == 0 ? n - 1 : k - 1), a1x, a1y, b1);
        line(I(k), a2x, a2y, b2);
        const double det = a1x * a2y - a1y * a2x;
        ux = (b1 * a2y - b2 * a1y) / det;
        uy = (a1x * b2 - a2x * b1) / det;
        return fabs(det) / (sqrt(a1x * a1x + a1y * a1y) * sqrt(a2x * a2x + a2y * a2y));
    }
    SDOT_HDI void vert(int k) const {
        if (k == ck) return;
        double ux, uy;
        solve(k, ux, uy);
        vx = c0x + ux;
        vy = c0y + uy;
        ck = k;
    }
    SDOT_HDI double X(int k) const {
        vert(k);
        return vx;
    }
    SDOT_HDI double Y(int k) const {
        vert(k);
        return vy;
    }
    // The FP32 topology is the FP64 one when: every FP64 vertex is near its
    // FP32 vertex, no two consecutive edges are nearly parallel, and every
    // FP64 edge runs the way its FP32 edge does and is not nearly of zero
    // length (a reversed or vanishing edge marks a vertex where four cells
    // nearly meet, whose topology depends on rounding).
    SDOT_HDI bool consistent() const {
        double vx0 = 0, vy0 = 0, px = 0, py = 0;
        float gx = 0, gy = 0;
        for (int k = 0; k <= n && n >= 2; ++k) {
            const int kk = k == n ? 0 : k;
            double ux, uy;
            if (k == n) {
                ux = vx0;
                uy = vy0;
            } else {
                const double sn = solve(kk, ux, uy);
                if (!(sn > 1e-6)) return false;
            }
            const float fx = poly.X(kk), fy = poly.Y(kk);
            const double sc = fabs(double(fx)) + fabs(double(fy)) + 1e-300;
            if (!(fabs(ux - fx) + fabs(uy - fy) <= 1e-4 * sc)) return false;
            if (k == 0) {
                vx0 = ux;
                vy0 = uy;
            } else {
                const double ex = ux - px, ey = uy - py;
                const double fex = double(fx) - gx, fey = double(fy) - gy;
                if (!(ex * fex + ey * fey > 0)) return false;
                if (fabs(ex) + fabs(ey) <= 1e-7 * (sc + fabs(px) + fabs(py))) return false;
            }
            px = ux;
            py = uy;
            gx = fx;
            gy = fy;
        }
        return true;
    }
};

// Per-cell work once the polygon of Dirac s is built (n vertices; -1: a
// capacity was exceeded, -2: a guard failed).  Returns false when a capacity
// was exceeded (the cell is then rebuilt by the next tier, which rewrites
// every output of it).
template <int MODE, bool BALL, class P>
SDOT_KFN bool finish_cell(const Cell2DArgs &A, long long s, const P &cell, int n, double *acc, int acc_st, Out &row,
                          Out &nbo) {
    const double c0x = A.pos[2 * s], c0y = A.pos[2 * s + 1], w0 = A.w[s];
    if (n == -2) {
        // failed guard: report a NaN cell, not an overflow
        if (A.mass) A.mass[s] = nan("");
        if (A.mass_c) A.mass_c[s] = nan("");
        if (A.ctd) A.ctd[2 * s] = A.ctd[2 * s + 1] = nan("");
        row.emit(int(s), 0.0);
        return true;
    }
    if (n < 0) return false;

    const double r = BALL ? sqrt(w0) : -1.0;
    if (MODE == DM_RASTER) {
        raster_cell<BALL>(A, s, cell, n, c0x, c0y, r);
        return true;
    }
    constexpr bool DIRECT = MODE == DM_SINGLE || MODE == DM_PERIODIC;
    using SinkT = Sink<DIRECT, P, MODE == DM_IMAGE6>;
    SinkT sink(cell, A.pos, c0x, c0y, BALL ? r : sqrt(w0), r, acc, acc_st, row);
    sink.n_diracs = A.n;
    sink.trans = A.trans;

    if (DIRECT && !BALL) {
        // reference order: fan from vertex 0, boundary items from edge (n-1 -> 0)
        double tr2 = 0;
        for (int i = 2; i < n; ++i) {
            const double ax = cell.X(0), ay = cell.Y(0);
            const double bx = cell.X(i - 1), by = cell.Y(i - 1), cx = cell.X(i), cy = cell.Y(i);
            const double t2 = ax * (by - cy) + bx * (cy - ay) + cx * (ay - by);
            tr2 += t2;
            const double lea = 0.5 * t2 * A.coeff;
            const double f = (1.0 / 3.0) * lea;
            sink.momx += f * (ax + bx + cx);
            sink.momy += f * (ay + by + cy);
            sink.mass_c += lea;
        }
        sink.mass = A.coeff * (tr2 * 0.5);
        sink.begin_piece(A.coeff);
        for (int i1 = 0, i0 = n - 1; i1 < n; i0 = i1++) {
            const double dx = cell.X(i1) - cell.X(i0), dy = cell.Y(i1) - cell.Y(i0);
            sink.line(i0, sqrt(dx * dx + dy * dy));
        }
    } else if (DIRECT) {
        sink.begin_piece(A.coeff);
        DiscClip<SinkT> dc(sink, c0x, c0y, r);
        stream_cell(cell, n, dc);
        sink.end_piece(dc.result_radius());
    } else {
        for (int k = 0; k < n; ++k) acc[k * acc_st] = -1.0;
        if (n > 0) {
            if (MODE == DM_IMAGE || MODE == DM_IMAGE6) {
                double xmin = cell.X(0), xmax = xmin, ymin = cell.Y(0), ymax = ymin;
                for (int k = 1; k < n; ++k) {
                    xmin = fmin(xmin, cell.X(k)); xmax = fmax(xmax, cell.X(k));
                    ymin = fmin(ymin, cell.Y(k)); ymax = fmax(ymax, cell.Y(k));
                }
                if (BALL) {
                    xmin = fmax(xmin, c0x - r); xmax = fmin(xmax, c0x + r);
                    ymin = fmax(ymin, c0y - r); ymax = fmin(ymax, c0y + r);
                }
                const double psx = (A.img_hi[0] - A.img_lo[0]) / A.img_nx;
                const double psy = (A.img_hi[1] - A.img_lo[1]) / A.img_ny;
                // pixels outside the cell's bounding box give empty pieces
                int ix0 = int(floor((xmin - A.img_lo[0]) / psx)), ix1 = int(floor((xmax - A.img_lo[0]) / psx));
                int iy0 = int(floor((ymin - A.img_lo[1]) / psy)), iy1 = int(floor((ymax - A.img_lo[1]) / psy));
                ix0 = max(ix0, 0); iy0 = max(iy0, 0);
                ix1 = min(ix1, A.img_nx - 1); iy1 = min(iy1, A.img_ny - 1);
                for (int iy = iy0; iy <= iy1; ++iy) {
                    const double y0 = A.img_lo[1] + psy * double(iy), y1 = A.img_lo[1] + psy * double(iy + 1);
                    for (int ix = ix0; ix <= ix1; ++ix) {
                        const double x0 = A.img_lo[0] + psx * double(ix), x1 = A.img_lo[0] + psx * double(ix + 1);
                        if (MODE == DM_IMAGE6)
                            sink.begin_piece_poly(A.img + (long long)iy * A.img_nx + ix,
                                                  (long long)A.img_nx * A.img_ny);
                        else
                            sink.begin_piece(A.img[(long long)iy * A.img_nx + ix]);
                        if (BALL && MODE == DM_IMAGE) {
                            DiscClip<SinkT> dc(sink, c0x, c0y, r);
                            AxisClip<DiscClip<SinkT>> c4(dc, 1, y1, -1.0, PID_OWN);
                            AxisClip<AxisClip<DiscClip<SinkT>>> c3(c4, 1, y0, 1.0, PID_OWN);
                            AxisClip<AxisClip<AxisClip<DiscClip<SinkT>>>> c2(c3, 0, x1, -1.0, PID_OWN);
                            AxisClip<AxisClip<AxisClip<AxisClip<DiscClip<SinkT>>>>> c1(c2, 0, x0, 1.0, PID_OWN);
                            stream_cell(cell, n, c1);
                            sink.end_piece(dc.result_radius());
                        } else {
                            AxisClip<SinkT> c4(sink, 1, y1, -1.0, PID_OWN);
                            AxisClip<AxisClip<SinkT>> c3(c4, 1, y0, 1.0, PID_OWN);
                            AxisClip<AxisClip<AxisClip<SinkT>>> c2(c3, 0, x1, -1.0, PID_OWN);
                            AxisClip<AxisClip<AxisClip<AxisClip<SinkT>>>> c1(c2, 0, x0, 1.0, PID_OWN);
                            stream_cell(cell, n, c1);
                            sink.end_piece(-1.0);
                        }
                    }
                }
            }
        }
        if (A.rows.cnt) {
            for (int i1 = 0, i0 = n - 1; i1 < n; i0 = i1++) {
                const double m = acc[i0 * acc_st];
                if (m < 0) continue;
                const int id = cell.I(i0);
                if (id < 0 || id >= A.n) {
                    guard_fail(A, 4, s, id);
                    continue;
                }
                const double dx = c0x - A.pos[2 * id], dy = c0y - A.pos[2 * id + 1];
                const double dist = sqrt(dx * dx + dy * dy);
                if (dist != 0) {
                    const double b = 0.5 * m / dist;
                    row.emit(id, -b);
                    sink.der0 += b;
                }
            }
        }
    }

    if (A.rows.cnt) {
        row.emit(int(s), sink.der0);
        if (!row.ok()) return false;
    }
    if (A.nb.cnt) {
        if (BALL) {
            NbSink<P> nbs(cell, nbo);
            DiscClip<NbSink<P>> dc(nbs, c0x, c0y, r);
            stream_cell(cell, n, dc);
        } else {
            for (int k = 0; k < n; ++k) nbo.emit(cell.I(k), 0.0);
        }
        if (!nbo.ok()) return false;
    }
    if (A.mass) A.mass[s] = sink.mass;
    if (A.mass_c) A.mass_c[s] = sink.mass_c;
    if (A.ctd) {
        const double d = sink.mass_c + (sink.mass_c == 0);
        A.ctd[2 * s] = sink.momx / d;
        A.ctd[2 * s + 1] = sink.momy / d;
    }
    return true;
}

// Hands cell s to the warp tier.  The list holds n entries and one launch
// appends each cell at most once; the bound check turns a count that was not
// reset between launches into an error instead of a write past the list.
__device__ void push_overflow(const Cell2DArgs &A, long long s) {
    const int k = atomicAdd(A.ovf_cnt, 1);
    if (k < A.n)
        A.ovf_list[k] = int(s);
    else
        flag_error(A.err, DE_CAPACITY);
}

// shared memory of the fast kernels, in half-doubles per vertex slot and
// thread beyond the polygon: the per-edge accumulators of the image mode
template <int MODE>
constexpr int smem_extra_halves() {
    return MODE == DM_IMAGE || MODE == DM_IMAGE6 ? 2 : 0;
}

template <int MODE, bool BALL>
// six blocks of T2D_MAX threads per SM: at most 85 registers per thread
__global__ void __launch_bounds__(T2D_MAX, 6) k_cells2d(const Cell2DArgs A) {
    extern __shared__ double smem[];
    constexpr int CAP = CAP_FAST_2D;
    const int t = threadIdx.x, T2D = blockDim.x;
    double *sx = smem;
    double *sy = sx + CAP * T2D;
    int *sid = reinterpret_cast<int *>(sy + CAP * T2D);
    double *extra = sy + CAP * T2D + (CAP * T2D + 1) / 2;
    PolyView<double> cell{sx + t, sy + t, sid + t, T2D, CAP};
    double *acc = extra + t;
    const long long s = blockIdx.x * (long long)T2D + t;
    if (s >= A.n) return;
    const int n = build_cell<MODE == DM_PERIODIC>(A, s, cell, CAP, A.pos[2 * s], A.pos[2 * s + 1], A.w[s]);
    SDOT_WORK_ADD(5, n > 0 ? n : 0);
    SDOT_WORK_ADD(6, 1);
    Out row(A.rows.cnt ? A.rows.col + s : nullptr, A.rows.cnt ? A.rows.val + s : nullptr, A.rows.stride, A.rows.cap);
    Out nbo(A.nb.cnt ? A.nb.col + s : nullptr, nullptr, A.nb.stride, A.nb.cap);
    if (finish_cell<MODE, BALL>(A, s, cell, n, acc, T2D, row, nbo)) {
        if (A.rows.cnt) A.rows.cnt[s] = row.cnt;
        if (A.nb.cnt) A.nb.cnt[s] = nbo.cnt;
    } else {
        push_overflow(A, s);
    }
}

// Fast tier of the mixed-precision path: FP32 build (polygon as floats in
// shared memory), FP64 re-clip of its vertices and FP64 integration.  Cells
// whose FP32 decisions were too close to call, whose topology does not
// re-clip cleanly, or that overflow the capacity go to the FP64 warp tier.
template <int MODE, bool BALL>
// six blocks of T2D_MAX threads per SM, as the FP64 kernel (4% faster on the
// 1M clustered mix than the unbounded 96 registers)
__global__ void __launch_bounds__(T2D_MAX, 6) k_cells2d_mixed(const Cell2DArgs A) {
    extern __shared__ double smem[];
    constexpr int CAP = CAP_FAST_2D;
    const int t = threadIdx.x, T2D = blockDim.x;
    float *sx = reinterpret_cast<float *>(smem);
    float *sy = sx + CAP * T2D;
    int *sid = reinterpret_cast<int *>(sy + CAP * T2D);
    double *extra = reinterpret_cast<double *>(sid + CAP * T2D);
    PolyView<float> cell{sx + t, sy + t, sid + t, T2D, CAP};
    double *acc = extra + t;
    const long long s = blockIdx.x * (long long)T2D + t;
    if (s >= A.n) return;
    const double c0x = A.pos[2 * s], c0y = A.pos[2 * s + 1], w0 = A.w[s];
    int n = build_cell_f32(A, s, cell, CAP, c0x, c0y, w0, true);
    if (n == -4) {
        n = build_cell_f32(A, s, cell, CAP, c0x, c0y, w0, false);
        if (n > 0) n = -3;  // only an empty cell is decided by the domain-wide FP32 walk
    }
    const ReclipView view{A, cell, n > 0 ? n : 0, c0x, c0y, w0};
    bool ok = n >= 0 || n == -2;
    if (n > 0 && !view.consistent()) ok = false;
    if (ok) {
        Out row(A.rows.cnt ? A.rows.col + s : nullptr, A.rows.cnt ? A.rows.val + s : nullptr, A.rows.stride,
                A.rows.cap);
        Out nbo(A.nb.cnt ? A.nb.col + s : nullptr, nullptr, A.nb.stride, A.nb.cap);
        ok = finish_cell<MODE, BALL>(A, s, view, n, acc, T2D, row, nbo);
        if (ok) {
            if (A.rows.cnt) A.rows.cnt[s] = row.cnt;
            if (A.nb.cnt) A.nb.cnt[s] = nbo.cnt;
        }
    }
    if (!ok) push_overflow(A, s);
}

// Polygon, accumulators and row buffers of one warp of the warp tier,
// contiguous (vertex k at index k) so that the lanes read 32 vertices at once.
struct WarpScratch {
    PolyView<double> cell;
    double *acc, *row_val;
    int *row_col, *nb_id;
    __device__ WarpScratch(double *base, int cap) {
        double *p = base;
        cell = PolyView<double>{p, p + cap, reinterpret_cast<int *>(p + 2 * cap), 1, cap};
        p += 3 * cap;
        acc = p;
        p += cap;
        row_val = p;
        p += cap + 1;
        row_col = reinterpret_cast<int *>(p);
        p += cap + 1;
        nb_id = reinterpret_cast<int *>(p);  // 2 cap ints
    }
};
// doubles of one warp's scratch: cell (3 cap), acc (cap), row values (cap + 1),
// row columns (cap + 1), ids (2 cap ints), rounded up
__host__ __device__ constexpr long long warp_scratch_doubles(int cap) {
    return (5LL * cap + 2LL * (cap + 1) + 31) / 32 * 32;
}

// Copies a finished row from scratch to its ELL slot or the side buffer.
__device__ bool commit(const Rows &R, long long s, const int *col, const double *val, long long st, int cnt) {
    if (cnt <= R.cap) {
        for (int k = 0; k < cnt; ++k) {
            R.col[k * R.stride + s] = col[k * st];
            if (R.val) R.val[k * R.stride + s] = val[k * st];
        }
    } else {
        const unsigned long long off = atomicAdd(R.side_used, (unsigned long long)cnt);
        if ((long long)(off + cnt) > R.side_cap) return false;  // the caller flags DE_SIDE
        R.side[s] = (long long)off;
        for (int k = 0; k < cnt; ++k) {
            R.side_col[off + k] = col[k * st];
            if (R.side_val) R.side_val[off + k] = val[k * st];
        }
    }
    R.cnt[s] = cnt;
    return true;
}

// Warp-per-cell build of one large cell (all lanes, same s): the walk of
// build_cell, with the eviction test and the plane cuts spread over the
// lanes, 32 vertices at a time.
template <bool PER = false>
__device__ int build_cell_coop(const Cell2DArgs &A, long long s, const PolyView<double> &cell, int cap, double c0x,
                               double c0y, double w0, int *wstack) {
    constexpr unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    int n = A.start_n;
    if (lane == 0) {
        for (int k = 0; k < n; ++k) {
            cell.X(k) = A.start_xy[2 * k];
            cell.Y(k) = A.start_xy[2 * k + 1];
            cell.I(k) = domain_id(k);
        }
    }
    __syncwarp();
    int visits = 0;
    // PER: one walk of the tree per translation after the untranslated one
    // (see build_cell)
    for (int sym = -1; sym < (PER ? A.ntrans : 0); ++sym) {
        const double tx = sym >= 0 ? A.trans[2 * sym] : 0.0, ty = sym >= 0 ? A.trans[2 * sym + 1] : 0.0;
        if (lane == 0) wstack[0] = 0;
        __syncwarp();
        int sp = 1;
        for (; sp > 0; ++visits) {
            if (visits > (PER ? (A.ntrans + 1) * A.max_nodes : A.max_nodes)) {
                if (lane == 0) flag_error(A.err, DE_ITER);
                return -1;
            }
            const int node = wstack[--sp];
            __syncwarp();
            const TreeNode<2> nd = A.nodes[SDOT_CHECK_IDX(node, A.max_nodes, 4)];
            const double lo0 = PER ? nd.lo[0] + tx : nd.lo[0], lo1 = PER ? nd.lo[1] + ty : nd.lo[1];
            const double hi0 = PER ? nd.hi[0] + tx : nd.hi[0], hi1 = PER ? nd.hi[1] + ty : nd.hi[1];
            bool need = false;
            for (int base = 0; base < n; base += 32) {
                const int k = base + lane;
                bool fail = false;
                if (k < n) {
                    const double px = cell.X(k), py = cell.Y(k);
                    const double qx = fmin(hi0, fmax(lo0, px));
                    const double qy = fmin(hi1, fmax(lo1, py));
                    const double lhs = (c0x - px) * (c0x - px) + (c0y - py) * (c0y - py) - w0;
                    const double rhs = (qx - px) * (qx - px) + (qy - py) * (qy - py) - nd.maxw;
                    fail = !(lhs <= rhs);
                }
                if (__any_sync(FULL, fail)) {
                    need = true;
                    break;
                }
            }
            if (!need) continue;
            if (nd.b < 0) {
                const int first = nd.a, nch = -nd.b;
                if (nch < 2 || nch > 4 || first < 1 || first + nch > A.max_nodes) {
                    if (lane == 0) guard_fail(A, 1, s, node);
                    return -2;
                }
                if (sp + nch > STACK) {
                    if (lane == 0) flag_error(A.err, DE_STACK);
                    return -1;
                }
                int ch[4];
                order_children<PER>(A, first, nch, c0x, c0y, tx, ty, ch);
                if (lane == 0) {
#pragma unroll
                    for (int c = 0; c < 4; ++c)
                        if (c < nch) wstack[sp + c] = ch[c];
                }
                __syncwarp();
                sp += nch;
            } else {
                if (nd.a < 0 || nd.b > A.n) {
                    if (lane == 0) guard_fail(A, 2, s, node);
                    return -2;
                }
                for (int j = nd.a; j < nd.b; ++j) {
                    if (j == s && sym < 0) continue;
                    const double c1x = PER ? A.pos[2 * j] + tx : A.pos[2 * j];
                    const double c1y = PER ? A.pos[2 * j + 1] + ty : A.pos[2 * j + 1];
                    const double w1 = A.w[j];
                    double ox, oy, nx, ny;
                    bisector(c0x, c0y, w0, c1x, c1y, w1, ox, oy, nx, ny);
                    n = plane_cut_warp(cell, n, cap, ox, oy, nx, ny, PER ? j + (sym + 1) * int(A.n) : j, true);
                    if (n <= 0) return n;
                }
            }
        }
    }
    return n;
}

// Cells that overflowed the fast tier: one warp per cell, polygon of up to
// CAP_HUGE_2D vertices in global scratch; lane 0 integrates the built cell.
template <int MODE, bool BALL>
__global__ void __launch_bounds__(128) k_cells2d_wtier(const Cell2DArgs A, double *scratch, int nwarps,
                                                       const int *list, const int *list_cnt) {
    constexpr int CAP = CAP_HUGE_2D;
    __shared__ int wstack[4][STACK];
    const int lane = threadIdx.x & 31, wb = threadIdx.x >> 5;
    const int gw = blockIdx.x * 4 + wb;
    if (gw >= nwarps) return;
    WarpScratch W(scratch + (long long)gw * warp_scratch_doubles(CAP), CAP);
    const int cnt = *list_cnt;
    for (int i = gw; i < cnt; i += nwarps) {
        const long long s = list[i];
        const int n = build_cell_coop<MODE == DM_PERIODIC>(A, s, W.cell, CAP, A.pos[2 * s], A.pos[2 * s + 1], A.w[s],
                                                           wstack[wb]);
        if (lane == 0) {
            Out row(A.rows.cnt ? W.row_col : nullptr, W.row_val, 1, CAP + 1);
            Out nbo(A.nb.cnt ? W.nb_id : nullptr, nullptr, 1, 2 * CAP);
            const bool built = finish_cell<MODE, BALL>(A, s, W.cell, n, W.acc, 1, row, nbo);
            bool ok = built;
            if (ok && A.rows.cnt) ok = commit(A.rows, s, W.row_col, W.row_val, 1, row.cnt);
            if (ok && A.nb.cnt) ok = commit(A.nb, s, W.nb_id, nullptr, 1, nbo.cnt);
            if (!ok) {
                atomicOr(A.err, built ? DE_SIDE : DE_CAPACITY);
                if (A.mass) A.mass[s] = nan("");
                if (A.rows.cnt) A.rows.cnt[s] = 0;
                if (A.nb.cnt) A.nb.cnt[s] = 0;
            }
        }
        __syncwarp();
    }
}

// The block size of the fast kernels is picked once per kernel variant and
// device by timing the candidates on the first evaluation large enough to
// tell them apart (the results do not depend on it: one thread builds one
// cell whatever the block).

template <int MODE, bool BALL>
size_t fast_smem(int bs, bool mixed) {
    constexpr int CAP = CAP_FAST_2D;
    const size_t extra = size_t(smem_extra_halves<MODE>()) * CAP * bs * 4;
    return mixed ? size_t(CAP) * bs * 12 + extra : size_t(CAP) * bs * 16 + size_t(CAP * bs + 1) / 2 * 8 + extra;
}

template <int MODE, bool BALL>
void launch_fast(const Cell2DArgs &a, int bs, cudaStream_t st) {
    const size_t smem = fast_smem<MODE, BALL>(bs, a.mixed != 0);
    if (a.mixed)
        k_cells2d_mixed<MODE, BALL><<<ceil_div(a.n, bs), bs, smem, st>>>(a);
    else
        k_cells2d<MODE, BALL><<<ceil_div(a.n, bs), bs, smem, st>>>(a);
    note_launch();
    SDOT_CUDA(cudaGetLastError());
}

// Every cell into the warp tier's list (domain polygons larger than the fast
// tier's polygons).
__global__ void k_all_cells(int *list, int *cnt, long long n) {
    const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (s < n) list[s] = int(s);
    if (s == 0) *cnt = int(n);
}

// Counters the fast kernel appends to: zeroed before every launch of it.
void reset_overflow(const Cell2DArgs &a, cudaStream_t st) {
    SDOT_CUDA(cudaMemsetAsync(a.ovf_cnt, 0, sizeof(int), st));
    if (a.rows.side_used) SDOT_CUDA(cudaMemsetAsync(a.rows.side_used, 0, sizeof(unsigned long long), st));
    if (a.nb.side_used) SDOT_CUDA(cudaMemsetAsync(a.nb.side_used, 0, sizeof(unsigned long long), st));
}

template <int MODE, bool BALL>
void launch_all(const Cell2DArgs &a, void *scratch, cudaStream_t st) {
    static PerDevice<int> attr_set;
    attr_set.once([] {
        SDOT_CUDA(cudaFuncSetAttribute(k_cells2d<MODE, BALL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       int(fast_smem<MODE, BALL>(T2D_MAX, false))));
        SDOT_CUDA(cudaFuncSetAttribute(k_cells2d_mixed<MODE, BALL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       int(fast_smem<MODE, BALL>(T2D_MAX, true))));
        // 72% of the shared memory capacity (164 KB: 16 warps of 64-thread
        // blocks) leaves the rest to L1 for the walk's tree, Diracs and stack;
        // measured 2% faster on the 1M clustered mix than the largest carveout
        SDOT_CUDA(cudaFuncSetAttribute(k_cells2d<MODE, BALL>, cudaFuncAttributePreferredSharedMemoryCarveout, 72));
    });
    if (a.start_n > CAP_FAST_2D) {
        // the starting polygon alone overflows the fast tier: every cell is
        // built by the warp tier (polygons of up to CAP_HUGE_2D vertices)
        reset_overflow(a, st);
        k_all_cells<<<ceil_div(a.n, 256), 256, 0, st>>>(a.ovf_list, a.ovf_cnt, a.n);
        note_launch();
        k_cells2d_wtier<MODE, BALL><<<WTIER_WARPS / 4, 128, 0, st>>>(a, static_cast<double *>(scratch), WTIER_WARPS,
                                                                      a.ovf_list, a.ovf_cnt);
        note_launch();
        SDOT_CUDA(cudaGetLastError());
        return;
    }
    static PerDevice<int> tuned[2];  // best block size per device: FP64, mixed
    PerDevice<int> &tu = tuned[a.mixed ? 1 : 0];
    int best = tu.get();
    if (!best && a.n >= (1 << 17)) {
        // time each candidate on this evaluation's cells; every output of the
        // trial runs is rewritten by the run that follows, and the overflow
        // counters are zeroed before each run
        const int cand[3] = {32, 64, 128};
        float best_ms = 0;
        cudaEvent_t e0, e1;
        SDOT_CUDA(cudaEventCreate(&e0));
        SDOT_CUDA(cudaEventCreate(&e1));
        for (int bs : cand) {
            reset_overflow(a, st);
            SDOT_CUDA(cudaEventRecord(e0, st));
            launch_fast<MODE, BALL>(a, bs, st);
            SDOT_CUDA(cudaEventRecord(e1, st));
            SDOT_CUDA(cudaEventSynchronize(e1));
            float ms = 0;
            SDOT_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            if (!best || ms < best_ms) {
                best = bs;
                best_ms = ms;
            }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        tu.set(best);
    }
    reset_overflow(a, st);
    launch_fast<MODE, BALL>(a, best ? best : 64, st);
    k_cells2d_wtier<MODE, BALL><<<WTIER_WARPS / 4, 128, 0, st>>>(a, static_cast<double *>(scratch), WTIER_WARPS,
                                                                  a.ovf_list, a.ovf_cnt);
    note_launch();
    SDOT_CUDA(cudaGetLastError());
}

}  // namespace

void cells2d_read_checks(unsigned long long out[3]) {
#ifdef SDOT_CHECKS
    SDOT_CUDA(cudaMemcpyFromSymbol(out, sdot_dbg_word, 3 * sizeof(unsigned long long)));
#else
    out[0] = out[1] = out[2] = 0;
#endif
}

void cells2d_read_work(unsigned long long out[8], bool reset) {
#ifdef SDOT_COUNT
    SDOT_CUDA(cudaMemcpyFromSymbol(out, sdot_work, 8 * sizeof(unsigned long long)));
    if (reset) {
        const unsigned long long z[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        SDOT_CUDA(cudaMemcpyToSymbol(sdot_work, z, sizeof z));
    }
#else
    (void)reset;
    for (int k = 0; k < 8; ++k) out[k] = 0;
#endif
}

size_t cells2d_scratch_bytes() {
    return size_t(warp_scratch_doubles(CAP_HUGE_2D)) * WTIER_WARPS * sizeof(double) + 256;
}

void cells2d_launch(const Cell2DArgs &a, void *scratch, cudaStream_t st) {
    if (a.n == 0) return;
    const bool ball = a.ball != 0;
    if (a.mode == DM_SINGLE) {
        if (ball) launch_all<DM_SINGLE, true>(a, scratch, st); else launch_all<DM_SINGLE, false>(a, scratch, st);
    } else if (a.mode == DM_PERIODIC) {
        // the mixed path has no periodic walk: the FP64 kernels run
        Cell2DArgs b = a;
        b.mixed = 0;
        if (ball) launch_all<DM_PERIODIC, true>(b, scratch, st); else launch_all<DM_PERIODIC, false>(b, scratch, st);
    } else if (a.mode == DM_IMAGE) {
        if (ball) launch_all<DM_IMAGE, true>(a, scratch, st); else launch_all<DM_IMAGE, false>(a, scratch, st);
    } else if (a.mode == DM_RASTER) {
        if (ball) launch_all<DM_RASTER, true>(a, scratch, st); else launch_all<DM_RASTER, false>(a, scratch, st);
    } else if (a.mode == DM_IMAGE6) {
        // the reference integrates no piecewise-quadratic density over disc arcs
        if (ball) throw CudaError{cudaErrorInvalidValue, "cells2d_launch: no disc clip with nb_coeffs = 6"};
        launch_all<DM_IMAGE6, false>(a, scratch, st);
    } else {
        throw CudaError{cudaErrorInvalidValue, "cells2d_launch: a domain of several shapes runs one pass per shape"};
    }
}

}  // namespace sdot
