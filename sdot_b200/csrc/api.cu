// C ABI of libsdot_b200.so (include/sdot_gpu.h): context, domain, evaluation.
#include "../../include/sdot_gpu.h"
#include "cell2d.cuh"
#include "cell3d.cuh"
#include "csr.cuh"
#include "derpos.cuh"
#include "geom2d.cuh"
#include "prims.cuh"
#include "solve.cuh"
#include "tree.cuh"

#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

using namespace sdot;

namespace sdot {
static std::atomic<unsigned long long> g_launches{0};
static thread_local unsigned long long *t_capture = nullptr;
void note_launch() {
    if (t_capture)
        ++*t_capture;
    else
        g_launches.fetch_add(1, std::memory_order_relaxed);
}
void note_launches(unsigned long long k) { g_launches.fetch_add(k, std::memory_order_relaxed); }
CaptureCount::CaptureCount() : prev(t_capture) { t_capture = &n; }
CaptureCount::~CaptureCount() { t_capture = prev; }
}  // namespace sdot

namespace {

struct BadArg : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct Unsupported : std::runtime_error {
    using std::runtime_error::runtime_error;
};

template <class T>
void dalloc(T *&p, size_t count) {
    if (p) cudaFree(p);
    p = nullptr;
    SDOT_CUDA(cudaMalloc(reinterpret_cast<void **>(&p), std::max<size_t>(count, 1) * sizeof(T) + 16));
}
template <class T>
void dfree(T *&p) {
    if (p) cudaFree(p);
    p = nullptr;
}

// A convex polygon of the domain: vertices (CCW) and the outward unit normal
// of the edge leaving each vertex.
struct Item2 {
    std::vector<double> xy, nrm;
    double coeff = 1;
    double area() const {
        // ConvexPolyhedron2::measure: fan from vertex 0 (ConvexPolyhedron2.tcc:1825-1832)
        size_t n = xy.size() / 2;
        double res = 0;
        for (size_t i = 2; i < n; ++i) {
            double ax = xy[0], ay = xy[1], bx = xy[2 * i - 2], by = xy[2 * i - 1], cx = xy[2 * i], cy = xy[2 * i + 1];
            res += ax * (by - cy) + bx * (cy - ay) + cx * (ay - by);
        }
        return 0.5 * res;
    }
};

// Host polygon used to build items with the same plane_cut as the kernels.
struct HostPoly {
    std::vector<double> x, y;
    std::vector<int> id;
    int n = 0;
    explicit HostPoly(int cap) : x(cap), y(cap), id(cap) {}
    PolyView<double> view() { return PolyView<double>{x.data(), y.data(), id.data(), 1}; }
};

const double kBoxNrm[4][2] = {{0, -1}, {1, 0}, {0, 1}, {-1, 0}};

// Domain polygons of more than CAP_FAST_2D vertices start every cell in the
// warp tier (polygons of up to CAP_HUGE_2D vertices); this leaves each cell
// room for 64 bisector edges.
constexpr int kMaxDomainVertices = CAP_HUGE_2D - 64;

// ConvexPolyhedron2( Box ) (ConvexPolyhedron2.tcc:76-106)
Item2 box_item(double x0, double y0, double x1, double y1, double coeff) {
    Item2 it;
    it.xy = {x0, y0, x1, y0, x1, y1, x0, y1};
    for (auto &n : kBoxNrm) { it.nrm.push_back(n[0]); it.nrm.push_back(n[1]); }
    it.coeff = coeff;
    return it;
}

// A convex polyhedron on the host, as faces (vertex loops counter-clockwise
// seen from outside): the domain shapes of 3D contexts, for their measures.
struct HostPoly3 {
    using P3 = std::array<double, 3>;
    std::vector<std::vector<P3>> faces;

    static HostPoly3 box(const double *lo, const double *hi) {
        HostPoly3 p;
        auto c = [&](int k) { return P3{(k & 1) ? hi[0] : lo[0], (k & 2) ? hi[1] : lo[1], (k & 4) ? hi[2] : lo[2]}; };
        const int f[6][4] = {{0, 4, 6, 2}, {1, 3, 7, 5}, {0, 1, 5, 4}, {2, 6, 7, 3}, {0, 2, 3, 1}, {4, 5, 7, 6}};
        for (auto &q : f) p.faces.push_back({c(q[0]), c(q[1]), c(q[2]), c(q[3])});
        return p;
    }
    // keeps a . x <= b
    void cut(const double *a, double b) {
        auto d = [&](const P3 &v) { return a[0] * v[0] + a[1] * v[1] + a[2] * v[2] - b; };
        bool removes = false;  // a plane that only touches the polyhedron changes nothing
        for (const auto &f : faces)
            for (const P3 &v : f) removes |= d(v) > 0;
        if (!removes) return;
        std::vector<std::vector<P3>> out;
        std::vector<P3> cap;  // points on the plane: the new face
        for (const auto &f : faces) {
            std::vector<P3> g;
            for (size_t i = 0; i < f.size(); ++i) {
                const P3 &u = f[i], &v = f[(i + 1) % f.size()];
                const double du = d(u), dv = d(v);
                if (du <= 0) g.push_back(u);
                if ((du < 0 && dv > 0) || (du > 0 && dv < 0)) {
                    const double t = du / (du - dv);
                    const P3 x{u[0] + t * (v[0] - u[0]), u[1] + t * (v[1] - u[1]), u[2] + t * (v[2] - u[2])};
                    g.push_back(x);
                    cap.push_back(x);
                } else if (du == 0) {
                    cap.push_back(u);
                }
            }
            if (g.size() >= 3) out.push_back(g);
        }
        if (cap.size() >= 3) {
            // order the new face's points counter-clockwise around a (outward)
            P3 c{0, 0, 0};
            for (const P3 &x : cap)
                for (int k = 0; k < 3; ++k) c[k] += x[k] / double(cap.size());
            const double na = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
            const P3 nn{a[0] / na, a[1] / na, a[2] / na};
            P3 e1{cap[0][0] - c[0], cap[0][1] - c[1], cap[0][2] - c[2]};
            const double l1 = std::sqrt(e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2]);
            if (l1 > 0) {
                for (double &x : e1) x /= l1;
                const P3 e2{nn[1] * e1[2] - nn[2] * e1[1], nn[2] * e1[0] - nn[0] * e1[2], nn[0] * e1[1] - nn[1] * e1[0]};
                std::vector<std::pair<double, P3>> ang;
                for (const P3 &x : cap) {
                    const P3 v{x[0] - c[0], x[1] - c[1], x[2] - c[2]};
                    ang.push_back({std::atan2(v[0] * e2[0] + v[1] * e2[1] + v[2] * e2[2],
                                              v[0] * e1[0] + v[1] * e1[1] + v[2] * e1[2]), x});
                }
                std::sort(ang.begin(), ang.end(), [](const auto &p, const auto &q) { return p.first < q.first; });
                std::vector<P3> face;
                for (const auto &pa : ang)
                    if (face.empty() || std::abs(pa.second[0] - face.back()[0]) + std::abs(pa.second[1] - face.back()[1]) +
                                                std::abs(pa.second[2] - face.back()[2]) > 0)
                        face.push_back(pa.second);
                if (face.size() >= 3) out.push_back(face);
            }
        }
        faces.swap(out);
    }
    // integral of c0 + c1 x + c2 y + c3 z + c4 xy + c5 xz + c6 yz + c7 xyz:
    // tetrahedra from the vertices' mean to each fan triangle, each by the
    // degree-3 five-point rule (weight -4/5 at the centroid, 9/20 at the four
    // points with barycentric coordinates (1/2, 1/6, 1/6, 1/6); P. Keast,
    // "Moderate-degree tetrahedral quadrature formulas", CMAME 55, 1986),
    // exact for this density
    double integrate(const double *c) const {
        P3 o{0, 0, 0};
        size_t cnt = 0;
        for (const auto &f : faces)
            for (const P3 &x : f) {
                for (int k = 0; k < 3; ++k) o[k] += x[k];
                ++cnt;
            }
        if (!cnt) return 0;
        for (double &x : o) x /= double(cnt);
        auto fv = [&](const P3 &x) {
            return c[0] + c[1] * x[0] + c[2] * x[1] + c[3] * x[2] + c[4] * x[0] * x[1] + c[5] * x[0] * x[2] +
                   c[6] * x[1] * x[2] + c[7] * x[0] * x[1] * x[2];
        };
        double res = 0;
        for (const auto &f : faces)
            for (size_t i = 1; i + 1 < f.size(); ++i) {
                const P3 v[4] = {o, f[0], f[i], f[i + 1]};
                const double ux = v[1][0] - o[0], uy = v[1][1] - o[1], uz = v[1][2] - o[2];
                const double vx = v[2][0] - o[0], vy = v[2][1] - o[1], vz = v[2][2] - o[2];
                const double wx = v[3][0] - o[0], wy = v[3][1] - o[1], wz = v[3][2] - o[2];
                const double vol = (ux * (vy * wz - vz * wy) - uy * (vx * wz - vz * wx) + uz * (vx * wy - vy * wx)) / 6;
                P3 g{0, 0, 0};
                for (int k = 0; k < 4; ++k)
                    for (int d = 0; d < 3; ++d) g[d] += 0.25 * v[k][d];
                double q = -0.8 * fv(g);
                for (int k = 0; k < 4; ++k) {
                    P3 x;
                    for (int d = 0; d < 3; ++d) x[d] = 0.5 * v[k][d] + (1.0 / 6.0) * (v[0][d] + v[1][d] + v[2][d] + v[3][d] - v[k][d]);
                    q += 0.45 * fv(x);
                }
                res += vol * q;
            }
        return res;
    }
};

}  // namespace

struct sdot_ctx {
    int dim = 2, precision = SDOT_FP64, device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::string last_error;
    long long max_per_leaf = 11;

    long long n = 0, cap = 0;
    double *d_pos = nullptr, *d_w = nullptr;
    DeviceTree<2> tree2;
    DeviceTree<3> tree3;
    // sorted -> caller order and its inverse, of the tree of this dimension
    const int *perm() const { return dim == 3 ? tree3.idx : tree2.idx; }
    const int *perm_inv() const { return dim == 3 ? tree3.inv : tree2.inv; }
    bool pos_dirty = true, w_dirty = true, dom_dirty = true, eval_dirty = true, nb_dirty = true;

    // domain (host side)
    std::vector<Item2> items;
    // a 3D domain shape: its box, cut by the half-spaces a . x <= b (4
    // doubles per plane; none for a box), and its density
    struct Item3 {
        double lo[3], hi[3], coeff;
        std::vector<double> planes;
    };
    std::vector<Item3> items3;
    double *d_planes3 = nullptr;       // every shape's planes, shape k from plane_off3[k]
    std::vector<int> plane_off3;
    bool planes3_dirty = true;
    bool has_poly = false;     // 3D multilinear density factor
    double poly3[8] = {1, 0, 0, 0, 0, 0, 0, 0};
    bool has_image = false;
    double img_lo[3] = {0, 0, 0}, img_hi[3] = {1, 1, 1};
    long long img_size[3] = {1, 1, 1};
    char *img_backup3 = nullptr;  // 3D voxel images: the kernels' per-warp face copies
    int img_ncoeffs = 1;
    std::vector<double> img_data;
    int ball = 0;
    // periodic copies of the Diracs (SpZGrid::translations, SpZGrid.h:53): x, y pairs
    std::vector<double> trans_h;
    double *d_trans = nullptr;
    // the kernel mode of a one-shape pass: with translations, the periodic walk
    int single_mode() const { return trans_h.empty() ? DM_SINGLE : DM_PERIODIC; }

    // domain (device side)
    int mode = DM_SINGLE;
    int start_n = 0;
    double coeff = 1;
    double *d_start = nullptr, *d_img = nullptr, *d_item_xy = nullptr, *d_item_nrm = nullptr, *d_item_coeff = nullptr;
    int *d_item_off = nullptr;

    // evaluation buffers
    long long ecap = 0;
    double *s_mass = nullptr, *s_mass_c = nullptr, *s_ctd = nullptr;
    double *o_mass = nullptr, *o_mass_c = nullptr, *o_ctd = nullptr;
    Rows rows, nb;             // Hessian rows, boundary id lists (sorted order)
    long long *cnt_orig = nullptr, *offsets = nullptr, *nb_offsets = nullptr;
    // Status words of one evaluation, kept together in device memory so that
    // one copy brings them all back (into the pinned mirror hstat).
    struct DevStatus {
        long long nnz;               // Hessian entries (the last CSR offset)
        unsigned long long n_void;   // empty cells
        unsigned err;                // DevErr bits
        int ovf;                     // cells handed to the overflow tier
        int guard[3];                // first failed guard (code, cell, value)
        int pad;
    };
    DevStatus *dstat = nullptr, *hstat = nullptr;
    int *ovf_list = nullptr, *ovf_cnt = nullptr;
    int *ovf_list2 = nullptr, *ovf_cnt2 = nullptr;  // 3D: third pass
    int *ovf_list3 = nullptr, *ovf_cnt3 = nullptr;  // 3D: fourth pass
    unsigned char *hint3 = nullptr;                  // 3D: pass of each cell last time
    bool hint_valid = false;
    void *scratch3 = nullptr;                        // 3D: third pass faces
    unsigned *err = nullptr;   // &dstat->err
    int *guard = nullptr;      // dstat->guard
    long long item_nv = 0;
    // device staging of the CSR columns / values and neighbour ids that go to
    // host buffers (int64 + double per entry), grown with nnz
    long long *stage_i = nullptr;
    double *stage_v = nullptr;
    long long stage_cap = 0;
    std::vector<int> item_off_h;  // vertex offsets of the shapes (several shapes)
    void *scratch = nullptr, *scan_tmp = nullptr;
    // several shapes: one cell pass per shape into these, summed into the above
    Rows rows_tmp;
    double *t_mass = nullptr, *t_mass_c = nullptr, *t_ctd = nullptr, *s_mom = nullptr;
    long long mcap = 0;
    long long nnz = 0, nb_total = 0;
    long long n_void = 0;
    int last_ovf = 0;
    unsigned last_err = 0;
    int last_guard[3] = {0, 0, 0};
    cudaEvent_t ev[4] = {};
    float times[3] = {0, 0, 0};

    ~sdot_ctx() {
        cudaSetDevice(device);
        tree2.release();
        tree3.release();
        dfree(d_pos); dfree(d_w);
        dfree(d_start); dfree(d_img); dfree(d_item_xy); dfree(d_item_nrm); dfree(d_item_coeff); dfree(d_item_off);
        dfree(d_trans);
        dfree(d_planes3);
        dfree(img_backup3);
        free_eval();
        free_newton();
        free_multi();
        for (auto &e : ev) if (e) cudaEventDestroy(e);
        if (hstat) cudaFreeHost(hstat);
        if (own_stream && stream) cudaStreamDestroy(stream);
    }

    void free_eval() {
        dfree(s_mass); dfree(s_mass_c); dfree(s_ctd); dfree(o_mass); dfree(o_mass_c); dfree(o_ctd);
        free_rows(rows);
        free_rows(nb);
        dfree(cnt_orig); dfree(offsets); dfree(nb_offsets);
        dfree(ovf_list); dfree(ovf_list2); dfree(ovf_cnt2); dfree(ovf_list3); dfree(ovf_cnt3); dfree(hint3);
        dfree(dstat);
        dfree(ras_buf);
        dfree(ras_nums);
        ras_cap = 0;
        ovf_cnt = nullptr;
        err = nullptr;
        guard = nullptr;
        dfree(stage_i); dfree(stage_v);
        stage_cap = 0;
        dfree(dp_off); dfree(dp_col); dfree(dp_val); dfree(dp_v);
        dp_ncap = dp_nnzcap = 0;
        if (scratch3) cudaFree(scratch3);
        scratch3 = nullptr;
        if (scratch) cudaFree(scratch);
        if (scan_tmp) cudaFree(scan_tmp);
        scratch = scan_tmp = nullptr;
        ecap = 0;
    }

    static void free_rows(Rows &r) {
        dfree(r.cnt); dfree(r.col); dfree(r.val); dfree(r.side); dfree(r.side_col); dfree(r.side_val);
        dfree(r.side_used);
        r = Rows();
    }
    // ELL of `width` slots per row plus a side buffer for the few longer rows
    static void alloc_rows(Rows &r, long long cap_n, int width, bool values) {
        free_rows(r);
        r.cap = width;
        r.stride = cap_n;
        r.side_cap = (1LL << 20) + cap_n / 8;
        dalloc(r.cnt, cap_n);
        dalloc(r.col, size_t(width) * cap_n);
        dalloc(r.side, cap_n);
        dalloc(r.side_col, r.side_cap);
        if (values) {
            dalloc(r.val, size_t(width) * cap_n);
            dalloc(r.side_val, r.side_cap);
        }
        dalloc(r.side_used, 1);
    }

    void reserve_eval() {
        if (ecap >= n && s_mass) return;
        free_eval();
        ecap = std::max<long long>(n, 1);
        dalloc(s_mass, ecap); dalloc(s_mass_c, ecap); dalloc(s_ctd, size_t(dim) * ecap);
        dalloc(o_mass, ecap); dalloc(o_mass_c, ecap); dalloc(o_ctd, size_t(dim) * ecap);
        alloc_rows(rows, ecap, dim == 3 ? ROWCAP_3D : ROWCAP_2D, true);
        dalloc(cnt_orig, ecap + 1);
        dalloc(offsets, ecap + 1);
        dalloc(ovf_list, ecap);
        dalloc(dstat, 1);
        ovf_cnt = &dstat->ovf;
        err = &dstat->err;
        guard = dstat->guard;
        if (!hstat) SDOT_CUDA(cudaMallocHost(reinterpret_cast<void **>(&hstat), sizeof(DevStatus)));
        if (dim == 3) {
            dalloc(ovf_list2, ecap);
            dalloc(ovf_cnt2, 1);
            dalloc(ovf_list3, ecap);
            dalloc(ovf_cnt3, 1);
            dalloc(hint3, ecap);
            hint_valid = false;
            SDOT_CUDA(cudaMalloc(&scratch3, cells3d_scratch_bytes()));
        }
        SDOT_CUDA(cudaMalloc(&scratch, cells2d_scratch_bytes()));
        SDOT_CUDA(cudaMalloc(&scan_tmp, scan_tmp_size(ecap + 1, sizeof(long long))));
    }

    void upload_domain() {
        if (!dom_dirty) return;
        if (has_image) {
            mode = img_ncoeffs == 6 ? DM_IMAGE6 : DM_IMAGE;
            std::vector<double> st = {img_lo[0], img_lo[1], img_hi[0], img_lo[1], img_hi[0], img_hi[1], img_lo[0], img_hi[1]};
            start_n = 4;
            dalloc(d_start, 8);
            SDOT_CUDA(cudaMemcpyAsync(d_start, st.data(), 8 * sizeof(double), cudaMemcpyHostToDevice, stream));
            dalloc(d_img, img_data.size());
            SDOT_CUDA(cudaMemcpyAsync(d_img, img_data.data(), img_data.size() * sizeof(double), cudaMemcpyHostToDevice, stream));
            coeff = 1;
        } else if (items.size() == 1) {
            // ConvexPolyhedronAssembly::englobing_convex_polyhedron with one item
            mode = single_mode();
            const Item2 &it = items[0];
            start_n = int(it.xy.size() / 2);
            dalloc(d_start, it.xy.size());
            SDOT_CUDA(cudaMemcpyAsync(d_start, it.xy.data(), it.xy.size() * sizeof(double), cudaMemcpyHostToDevice, stream));
            coeff = it.coeff;
        } else if (items.size() > 1) {
            // englobing box inflated by its own size on each side (ConvexPolyhedronAssembly.tcc:60-92)
            mode = DM_MULTI;
            double mn[2] = {std::numeric_limits<double>::max(), std::numeric_limits<double>::max()};
            double mx[2] = {-std::numeric_limits<double>::max(), -std::numeric_limits<double>::max()};
            std::vector<int> off = {0};
            std::vector<double> xy, nrm, co;
            for (const Item2 &it : items) {
                for (size_t k = 0; k < it.xy.size(); ++k) {
                    mn[k % 2] = std::min(mn[k % 2], it.xy[k]);
                    mx[k % 2] = std::max(mx[k % 2], it.xy[k]);
                }
                xy.insert(xy.end(), it.xy.begin(), it.xy.end());
                nrm.insert(nrm.end(), it.nrm.begin(), it.nrm.end());
                off.push_back(int(xy.size() / 2));
                co.push_back(it.coeff);
            }
            double dx = mx[0] - mn[0], dy = mx[1] - mn[1];
            Item2 eb = box_item(mn[0] - dx, mn[1] - dy, mx[0] + dx, mx[1] + dy, 1.0);
            start_n = 4;
            dalloc(d_start, 8);
            SDOT_CUDA(cudaMemcpyAsync(d_start, eb.xy.data(), 8 * sizeof(double), cudaMemcpyHostToDevice, stream));
            item_nv = off.back();
            item_off_h = off;
            for (size_t k = 0; k + 1 < off.size(); ++k)
                if (off[k + 1] - off[k] > kMaxDomainVertices)
                    throw Unsupported("a domain shape has more than " + std::to_string(kMaxDomainVertices) +
                                      " vertices");
            dalloc(d_item_off, off.size());
            SDOT_CUDA(cudaMemcpyAsync(d_item_off, off.data(), off.size() * sizeof(int), cudaMemcpyHostToDevice, stream));
            dalloc(d_item_xy, xy.size());
            SDOT_CUDA(cudaMemcpyAsync(d_item_xy, xy.data(), xy.size() * sizeof(double), cudaMemcpyHostToDevice, stream));
            dalloc(d_item_nrm, nrm.size());
            SDOT_CUDA(cudaMemcpyAsync(d_item_nrm, nrm.data(), nrm.size() * sizeof(double), cudaMemcpyHostToDevice, stream));
            dalloc(d_item_coeff, co.size());
            SDOT_CUDA(cudaMemcpyAsync(d_item_coeff, co.data(), co.size() * sizeof(double), cudaMemcpyHostToDevice, stream));
        } else {
            throw BadArg("no domain: call sdot_add_box_shape (or another add_..._shape) first");
        }
        if (start_n > kMaxDomainVertices)
            throw Unsupported("the domain polygon has more than " + std::to_string(kMaxDomainVertices) + " vertices");
        dom_dirty = false;
    }

    Cell2DArgs args() {
        Cell2DArgs a;
        a.n = n;
        a.pos = tree2.pos;
        a.w = tree2.w;
        a.nodes = tree2.nodes;
        a.max_nodes = tree2.max_nodes;
        a.guard = guard;
        a.item_nv = item_nv;
        a.start_n = start_n;
        a.start_xy = d_start;
        a.coeff = coeff;
        a.mode = mode;
        a.mixed = precision == SDOT_MIXED;
        a.ball = ball;
        a.img_lo[0] = img_lo[0]; a.img_lo[1] = img_lo[1];
        a.img_hi[0] = img_hi[0]; a.img_hi[1] = img_hi[1];
        a.img_nx = int(img_size[0]);
        a.img_ny = int(img_size[1]);
        a.img = d_img;
        a.nitems = int(items.size());
        a.item_off = d_item_off;
        a.item_xy = d_item_xy;
        a.item_nrm = d_item_nrm;
        a.item_coeff = d_item_coeff;
        a.ovf_list = ovf_list;
        a.ovf_cnt = ovf_cnt;
        a.err = err;
        a.ntrans = int(trans_h.size() / 2);
        a.trans = d_trans;
        return a;
    }

    // the domain is one the kernels handle; uploads the 2D one
    void check_domain() {
        if (dim == 3 && has_image) {
            if (ball) throw Unsupported("no ball cut in 3D (the reference's ConvexPolyhedron3::ball_cut is a TODO)");
            if (has_poly) throw Unsupported("a multilinear density factor with a voxel image is not available");
            if (dom_dirty) {
                dalloc(d_img, img_data.size());
                SDOT_CUDA(cudaMemcpy(d_img, img_data.data(), img_data.size() * sizeof(double), cudaMemcpyHostToDevice));
                if (!img_backup3) dalloc(img_backup3, cells3d_image_backup_bytes());
                dom_dirty = false;
            }
            return;
        }
        if (dim == 3) {
            if (items3.empty()) throw BadArg("no domain: call sdot_add_box_shape (or another add_..._shape) first");
            if (ball) throw Unsupported("no ball cut in 3D (the reference's ConvexPolyhedron3::ball_cut is a TODO)");
            if (!trans_h.empty()) throw Unsupported("periodic translations are available in 2D only");
            if (planes3_dirty) {
                std::vector<double> all;
                plane_off3.assign(1, 0);
                for (const Item3 &it : items3) {
                    all.insert(all.end(), it.planes.begin(), it.planes.end());
                    plane_off3.push_back(int(all.size() / 4));
                }
                dalloc(d_planes3, all.size());
                if (!all.empty())
                    SDOT_CUDA(cudaMemcpy(d_planes3, all.data(), all.size() * sizeof(double), cudaMemcpyHostToDevice));
                planes3_dirty = false;
            }
            return;
        }
        if (!trans_h.empty() && (long long)(trans_h.size() / 2 + 1) * n >= (1LL << 31))
            throw Unsupported("(translations + 1) x Diracs must stay below 2^31 (cut ids are 32-bit)");
        if (!trans_h.empty() && has_image)
            throw Unsupported("periodic translations with an image density are not available in this build");
        if (has_image && img_ncoeffs == 6 && ball)
            throw Unsupported("no ball cut with a piecewise-quadratic image (the reference's Polynomial<6> arc "
                              "integrals are a TODO)");
        upload_domain();
    }

    void reserve_multi() {
        if (mcap >= n && t_mass) return;
        free_multi();
        mcap = std::max<long long>(n, 1);
        alloc_rows(rows_tmp, mcap, dim == 3 ? ROWCAP_3D : ROWCAP_2D, true);
        dalloc(t_mass, mcap); dalloc(t_mass_c, mcap); dalloc(t_ctd, size_t(dim) * mcap); dalloc(s_mom, size_t(dim) * mcap);
    }
    void free_multi() {
        free_rows(rows_tmp);
        dfree(t_mass); dfree(t_mass_c); dfree(t_ctd); dfree(s_mom);
        mcap = 0;
    }

    // ConvexPolyhedronAssembly::for_each_intersection (ConvexPolyhedronAssembly.tcc:132-142)
    // sums over the shapes the integrals of cell ∩ shape.  Here: one cell
    // pass per shape, with the shape itself as the starting polygon (the
    // cell ∩ shape is the same convex set), summed: masses and centroid
    // moments added, Hessian rows appended (equal columns are merged by the
    // row assembly, as the reference merges its per-piece entries).
    void evaluate_multi() {
        reserve_multi();
        SDOT_CUDA(cudaMemsetAsync(s_mass, 0, size_t(n) * sizeof(double), stream));
        SDOT_CUDA(cudaMemsetAsync(s_mass_c, 0, size_t(n) * sizeof(double), stream));
        SDOT_CUDA(cudaMemsetAsync(s_mom, 0, size_t(2 * n) * sizeof(double), stream));
        rows_clear(rows, n, stream);
        SDOT_CUDA(cudaMemsetAsync(rows.side_used, 0, sizeof(unsigned long long), stream));
        for (size_t k = 0; k + 1 < item_off_h.size(); ++k) {
            Cell2DArgs a = args();
            a.mode = single_mode();
            a.start_n = item_off_h[k + 1] - item_off_h[k];
            a.start_xy = d_item_xy + 2 * item_off_h[k];
            a.coeff = items[k].coeff;
            a.mass = t_mass;
            a.mass_c = t_mass_c;
            a.ctd = t_ctd;
            a.rows = rows_tmp;
            cells2d_launch(a, scratch, stream);
            accum_pass(s_mass, s_mass_c, s_mom, t_mass, t_mass_c, t_ctd, n, 2, stream);
            rows_append(rows, rows_tmp, n, err, stream);
        }
        centroids_final(s_ctd, s_mom, s_mass_c, n, 2, stream);
    }

    // The 3D counterpart: one pass per shape (the shape's box cut by its
    // planes as the starting polyhedron), summed.  The cells' pass hints
    // belong to one starting polyhedron, so these passes neither use nor
    // record them.
    void evaluate_multi3() {
        reserve_multi();
        SDOT_CUDA(cudaMemsetAsync(s_mass, 0, size_t(n) * sizeof(double), stream));
        SDOT_CUDA(cudaMemsetAsync(s_mass_c, 0, size_t(n) * sizeof(double), stream));
        SDOT_CUDA(cudaMemsetAsync(s_mom, 0, size_t(3 * n) * sizeof(double), stream));
        rows_clear(rows, n, stream);
        SDOT_CUDA(cudaMemsetAsync(rows.side_used, 0, sizeof(unsigned long long), stream));
        for (size_t k = 0; k < items3.size(); ++k) {
            Cell3DArgs a = args3(int(k));
            a.hint = nullptr;
            a.use_hint = 0;
            a.mass = t_mass;
            a.ctd = t_ctd;
            a.rows = rows_tmp;
            cells3d_launch(a, scratch3, stream);
            accum_pass(s_mass, s_mass_c, s_mom, t_mass, t_mass, t_ctd, n, 3, stream);
            rows_append(rows, rows_tmp, n, err, stream);
        }
        centroids_final(s_ctd, s_mom, s_mass_c, n, 3, stream);
        hint_valid = false;
    }

    // arguments of a pass over shape k of the 3D domain (k = -1: the box
    // englobing every shape, inflated by its size as
    // ConvexPolyhedronAssembly::englobing_convex_polyhedron makes it, density 1)
    Cell3DArgs args3(int k = 0) {
        Cell3DArgs a;
        a.n = n;
        a.pos = tree3.pos;
        a.w = tree3.w;
        a.nodes = tree3.nodes;
        a.max_nodes = tree3.max_nodes;
        if (has_image) {
            // ScaledImage: the cells start from the image box
            for (int d = 0; d < 3; ++d) {
                a.box_lo[d] = a.img_lo[d] = img_lo[d];
                a.box_hi[d] = a.img_hi[d] = img_hi[d];
                a.img_n[d] = int(img_size[d]);
            }
            a.img = d_img;
            a.img_backup = img_backup3;
        } else if (k >= 0) {
            for (int d = 0; d < 3; ++d) {
                a.box_lo[d] = items3[k].lo[d];
                a.box_hi[d] = items3[k].hi[d];
            }
            a.coeff = items3[k].coeff;
            a.nplanes = plane_off3[k + 1] - plane_off3[k];
            a.planes = a.nplanes ? d_planes3 + 4 * plane_off3[k] : nullptr;
        } else {
            for (int d = 0; d < 3; ++d) {
                double lo = items3[0].lo[d], hi = items3[0].hi[d];
                for (const Item3 &it : items3) {
                    lo = std::min(lo, it.lo[d]);
                    hi = std::max(hi, it.hi[d]);
                }
                a.box_lo[d] = lo - (hi - lo);
                a.box_hi[d] = hi + (hi - lo);
            }
            a.coeff = 1.0;
        }
        a.has_poly = has_poly ? 1 : 0;
        for (int k = 0; k < 8; ++k) a.poly[k] = poly3[k];
        a.ovf_list = ovf_list;
        a.ovf_cnt = ovf_cnt;
        a.ovf_list2 = ovf_list2;
        a.ovf_cnt2 = ovf_cnt2;
        a.ovf_list3 = ovf_list3;
        a.ovf_cnt3 = ovf_cnt3;
        a.hint = hint3;
        a.use_hint = hint_valid ? 1 : 0;
        a.err = err;
        a.guard = guard;
        return a;
    }

    void ensure_tree() {
        if (n == 0) throw BadArg("no Diracs: call sdot_set_diracs first");
        if (pos_dirty) {
            if (dim == 3) {
                tree3.max_per_leaf = int(max_per_leaf);
                tree3.build(d_pos, d_w, n, stream);
                hint_valid = false;  // a new tree order: the hints no longer apply
            } else {
                tree2.max_per_leaf = int(max_per_leaf);
                tree2.build(d_pos, d_w, n, stream);
            }
            pos_dirty = w_dirty = false;
        } else if (w_dirty) {
            if (dim == 3)
                tree3.update_weights(d_w, stream);
            else
                tree2.update_weights(d_w, stream);
            w_dirty = false;
        }
    }

    int evaluate() {
        if (!eval_dirty) return finish_status();
        check_domain();
        reserve_eval();
        if (!ev[0]) for (auto &e : ev) SDOT_CUDA(cudaEventCreate(&e));
        SDOT_CUDA(cudaMemsetAsync(dstat, 0, sizeof(DevStatus), stream));
        SDOT_CUDA(cudaEventRecord(ev[0], stream));
        ensure_tree();
        SDOT_CUDA(cudaEventRecord(ev[1], stream));
        if (dim == 3 && items3.size() > 1 && !has_image) {
            evaluate_multi3();
        } else if (dim == 3) {
            Cell3DArgs a = args3(0);
            a.mass = s_mass;
            a.ctd = s_ctd;
            a.rows = rows;
            cells3d_launch(a, scratch3, stream);
            hint_valid = true;  // every cell of this tree order now has a pass hint
            // get_centroids' mass is the integral itself in 3D
            SDOT_CUDA(cudaMemcpyAsync(s_mass_c, s_mass, size_t(n) * sizeof(double), cudaMemcpyDeviceToDevice, stream));
        } else if (mode == DM_MULTI) {
            evaluate_multi();
        } else {
            Cell2DArgs a = args();
            a.mass = s_mass;
            a.mass_c = s_mass_c;
            a.ctd = s_ctd;
            a.rows = rows;
            cells2d_launch(a, scratch, stream);
        }
        SDOT_CUDA(cudaEventRecord(ev[2], stream));
        csr_sort_merge(rows, n, perm(), cnt_orig, dim == 2, stream);
        scan_exclusive_total<long long>(cnt_orig, offsets, n, scan_tmp, stream);
        unpermute(s_mass, o_mass, n, 1, perm(), stream);
        unpermute(s_mass_c, o_mass_c, n, 1, perm(), stream);
        unpermute(s_ctd, o_ctd, n, dim, perm(), stream);
        SDOT_CUDA(cudaEventRecord(ev[3], stream));
        // the status block (nnz, empty cells, error bits, overflow count,
        // guard) comes back in one copy
        SDOT_CUDA(cudaMemcpyAsync(&dstat->nnz, offsets + n, sizeof(long long), cudaMemcpyDeviceToDevice, stream));
        count_zeros(s_mass, n, &dstat->n_void, stream);
        SDOT_CUDA(cudaMemcpyAsync(hstat, dstat, sizeof(DevStatus), cudaMemcpyDeviceToHost, stream));
        SDOT_CUDA(cudaStreamSynchronize(stream));
        nnz = hstat->nnz;
        n_void = (long long)hstat->n_void;
        last_err = hstat->err;
        last_ovf = hstat->ovf;
        for (int k = 0; k < 3; ++k) last_guard[k] = hstat->guard[k];
        SDOT_CUDA(cudaEventElapsedTime(&times[0], ev[0], ev[1]));
        SDOT_CUDA(cudaEventElapsedTime(&times[1], ev[1], ev[2]));
        SDOT_CUDA(cudaEventElapsedTime(&times[2], ev[2], ev[3]));
        if ((last_err & DE_SIDE) && !(last_err & (DE_CAPACITY | DE_DEGEN)) && side_retries < 4) {
            // long rows outgrew the side buffer: grow it and evaluate again
            // (not when the evaluation failed anyway)
            ++side_retries;
            grow_side(rows);
            if ((dim != 3 && mode == DM_MULTI) || (dim == 3 && items3.size() > 1)) grow_side(rows_tmp);
            const int st = evaluate();
            side_retries = 0;
            return st;
        }
        eval_dirty = false;
        return finish_status();
    }

    int side_retries = 0;
    // a side buffer four times larger (the ELL part is kept)
    static void grow_side(Rows &r) {
        if (!r.side_col) return;
        r.side_cap *= 4;
        dalloc(r.side_col, r.side_cap);
        if (r.side_val) dalloc(r.side_val, r.side_cap);
    }

    int finish_status() {
        if (last_err & DE_ITER) {
            last_error = "a tree traversal visited more nodes than the tree holds (inconsistent tree)";
            return SDOT_ITER_CAP;
        }
        if (last_err & DE_CAPACITY) {
            last_error = dim == 3 ? "a cell exceeded the maximum polyhedron capacity (256 faces of 128 vertices)"
                                  : "a cell exceeded the maximum polygon capacity (1024 vertices)";
            return SDOT_CAPACITY;
        }
        if (last_err & DE_SIDE) {
            last_error = "long Hessian rows or neighbour lists exceeded the side buffer after it was grown";
            return SDOT_CAPACITY;
        }
        if (last_err & DE_DEGEN) {
            last_error = "a 3D cut met degenerate geometry (the affected cells are NaN)";
            return SDOT_CAPACITY;
        }
        if (last_err & DE_GUARD) {
            last_error = "inconsistent input or tree (guard " + std::to_string(last_guard[0]) + " at cell " +
                         std::to_string(last_guard[1]) + ", value " + std::to_string(last_guard[2]) + ")";
            return SDOT_BAD_ARG;
        }
        if (last_err & DE_STACK) {
            last_error = "traversal stack overflow";
            return SDOT_CAPACITY;
        }
        return SDOT_OK;
    }

    void evaluate_neighbors() {
        if (!nb_dirty) return;
        evaluate();
        if (!nb.cnt || nb.stride < ecap) alloc_rows(nb, ecap, dim == 3 ? NBCAP_3D : NBCAP_2D, false);
        if (!nb_offsets) dalloc(nb_offsets, ecap + 1);
        for (int attempt = 0;; ++attempt) {
            SDOT_CUDA(cudaMemsetAsync(err, 0, sizeof(unsigned), stream));
            if (dim == 3) {
                // several shapes: the traversal cell in the englobing box
                Cell3DArgs a = args3(items3.size() > 1 && !has_image ? -1 : 0);
                a.img = nullptr;  // the traversal cell, before any intersection
                if (items3.size() > 1 && !has_image) {
                    a.hint = nullptr;
                    a.use_hint = 0;
                }
                a.nb = nb;
                cells3d_launch(a, scratch3, stream);
            } else {
                // several shapes: the cut ids of the traversal cell in the
                // englobing box (the cell the reference's callback receives)
                Cell2DArgs a = args();
                if (mode == DM_MULTI) {
                    a.mode = single_mode();
                    a.coeff = 1.0;
                }
                a.nb = nb;
                cells2d_launch(a, scratch, stream);
            }
            unsigned e = 0;
            SDOT_CUDA(cudaMemcpyAsync(&e, err, sizeof(unsigned), cudaMemcpyDeviceToHost, stream));
            SDOT_CUDA(cudaStreamSynchronize(stream));
            if (!(e & DE_SIDE) || attempt >= 4) break;
            grow_side(nb);  // long id lists outgrew the side buffer
        }
        nb_counts(nb, n, perm(), cnt_orig, stream);
        scan_exclusive_total<long long>(cnt_orig, nb_offsets, n, scan_tmp, stream);
        SDOT_CUDA(cudaMemcpyAsync(&nb_total, nb_offsets + n, sizeof(long long), cudaMemcpyDeviceToHost, stream));
        SDOT_CUDA(cudaStreamSynchronize(stream));
        nb_dirty = false;
    }

    // get_image_integrals / get_image_of_cell_nums (get_image_integrals.h:16-78,
    // get_image_of_cell_nums.h:13-80): every cell (each piece cell ∩ shape
    // with its density, or cell ∩ disc) integrated over the pixels of the
    // raster [lo, hi] of nx x ny pixels; results in ras_buf (device, nx * ny *
    // 3 doubles) or ras_nums (device, nx * ny int64)
    double *ras_buf = nullptr;
    long long *ras_nums = nullptr;
    long long ras_cap = 0;
    void rasterize(const double *lo, const double *hi, long long nx, long long ny, bool nums) {
        if (dim != 2) throw Unsupported("image integrals are available in 2D");
        if (nx <= 0 || ny <= 0 || nx * ny > (1LL << 31)) throw BadArg("bad raster size");
        if (!(hi[0] > lo[0]) || !(hi[1] > lo[1])) throw BadArg("bad raster corners");
        check_domain();
        if (mode == DM_IMAGE || mode == DM_IMAGE6)
            throw Unsupported("image integrals over an image density are not available in this build");
        if (!trans_h.empty()) throw Unsupported("image integrals with periodic translations are not available");
        reserve_eval();
        ensure_tree();
        const long long np = nx * ny;
        if (ras_cap < np) {
            dalloc(ras_buf, size_t(3 * np));
            dalloc(ras_nums, size_t(np));
            ras_cap = np;
        }
        if (nums)
            SDOT_CUDA(cudaMemsetAsync(ras_nums, 0xff, size_t(np) * sizeof(long long), stream));  // -1
        else
            SDOT_CUDA(cudaMemsetAsync(ras_buf, 0, size_t(3 * np) * sizeof(double), stream));
        SDOT_CUDA(cudaMemsetAsync(dstat, 0, sizeof(DevStatus), stream));
        Cell2DArgs a = args();
        a.mixed = 0;
        a.ras = nums ? nullptr : ras_buf;
        a.ras_nums = nums ? ras_nums : nullptr;
        a.perm = perm();
        for (int d = 0; d < 2; ++d) {
            a.ras_lo[d] = lo[d];
            a.ras_hi[d] = hi[d];
        }
        a.ras_nx = int(nx);
        a.ras_ny = int(ny);
        if (mode == DM_MULTI) {
            // one pass per shape, with the shape as the starting polygon and
            // its density (the pieces of ConvexPolyhedronAssembly::for_each_intersection)
            for (size_t k = 0; k + 1 < item_off_h.size(); ++k) {
                Cell2DArgs b = a;
                b.mode = DM_RASTER;
                b.start_n = item_off_h[k + 1] - item_off_h[k];
                b.start_xy = d_item_xy + 2 * item_off_h[k];
                b.coeff = items[k].coeff;
                cells2d_launch(b, scratch, stream);
            }
        } else {
            a.mode = DM_RASTER;
            cells2d_launch(a, scratch, stream);
        }
        SDOT_CUDA(cudaMemcpyAsync(hstat, dstat, sizeof(DevStatus), cudaMemcpyDeviceToHost, stream));
        SDOT_CUDA(cudaStreamSynchronize(stream));
        last_err = hstat->err;
        for (int k = 0; k < 3; ++k) last_guard[k] = hstat->guard[k];
    }

    void copy_out(void *dst, const void *src, size_t bytes, int mem_space) {
        SDOT_CUDA(cudaMemcpyAsync(dst, src, bytes, mem_space == SDOT_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                                  stream));
    }

    void mark_dirty() { eval_dirty = nb_dirty = true; }

    // staging buffers of at least `count` entries (25% headroom when grown)
    // host-side outputs of the position derivatives: device staging kept
    // and grown like the Hessian's (3 n + 1 offsets, nnz entries, 3 n values)
    long long *dp_off = nullptr, *dp_col = nullptr;
    double *dp_val = nullptr, *dp_v = nullptr;
    long long dp_ncap = 0, dp_nnzcap = 0;
    void reserve_derpos(long long nn, long long nnz) {
        if (nn > dp_ncap || !dp_off) {
            const long long c = nn + nn / 4 + 16;
            dalloc(dp_off, size_t(3 * c + 1));
            dalloc(dp_v, size_t(3 * c));
            dp_ncap = c;
        }
        if (nnz > dp_nnzcap || !dp_col) {
            const long long c = nnz + nnz / 4 + 1024;
            dalloc(dp_col, size_t(c));
            dalloc(dp_val, size_t(c));
            dp_nnzcap = c;
        }
    }

    void reserve_stage(long long count) {
        if (count <= stage_cap && stage_i) return;
        const long long cap2 = count + count / 4 + 1024;
        dalloc(stage_i, size_t(cap2));
        dalloc(stage_v, size_t(cap2));
        stage_cap = cap2;
    }

    // ---- Newton on the weights (OptimalTransportSolver::solve, .tcc:27-119)
    long long ncap = 0;
    double *t_orig = nullptr, *t_sorted = nullptr, *w_old = nullptr, *dir = nullptr, *rhs = nullptr;
    double *pcg_buf = nullptr, *red = nullptr, *mg_buf = nullptr;
    PcgWork pcg;
    // FP32 solves with FP64 refinement: FP32 copies of the Hessian values,
    // FP32 work vectors and multilevel storage, the refinement's residual
    double *pcg32_buf = nullptr, *mg32_buf = nullptr, *ref_buf = nullptr;
    float *val32 = nullptr, *side32 = nullptr;
    long long side32_cap = 0, f32cap = 0;
    PcgWorkT<float> pcg32;

    void free_newton() {
        dfree(t_orig); dfree(t_sorted); dfree(w_old); dfree(dir); dfree(rhs); dfree(pcg_buf); dfree(red); dfree(mg_buf);
        dfree(pcg32_buf); dfree(mg32_buf); dfree(ref_buf); dfree(val32); dfree(side32);
        side32_cap = f32cap = 0;
        ncap = 0;
    }
    void reserve_fp32() {
        if (f32cap < n || !val32) {
            const long long c = std::max<long long>(n, 1);
            dalloc(pcg32_buf, pcg_work_doubles(c));
            dalloc(mg32_buf, mg_work_doubles(c, dim == 3 ? 128 : 64));
            dalloc(ref_buf, size_t(2 * c));
            dalloc(val32, size_t(rows.cap) * size_t(rows.stride));
            pcg_bind(pcg32, pcg32_buf, c);
            pcg32.mg = mg32_buf;
            pcg32.mg_cap = dim == 3 ? 128 : 64;
            pcg32.mg_doubles = mg_work_doubles(c, pcg32.mg_cap);
            f32cap = c;
        }
        if (side32_cap < rows.side_cap || !side32) {
            dalloc(side32, size_t(rows.side_cap));
            side32_cap = rows.side_cap;
        }
    }
    void reserve_newton() {
        if (ncap >= n && t_orig) return;
        free_newton();
        ncap = std::max<long long>(n, 1);
        dalloc(t_orig, ncap); dalloc(t_sorted, ncap); dalloc(w_old, ncap); dalloc(dir, ncap); dalloc(rhs, ncap);
        dalloc(pcg_buf, pcg_work_doubles(ncap));
        dalloc(mg_buf, mg_work_doubles(ncap, dim == 3 ? 128 : 64));
        dalloc(red, 3 * PCG_BLOCKS + 8);
        pcg_bind(pcg, pcg_buf, ncap);
        pcg.mg = mg_buf;
        pcg.mg_cap = dim == 3 ? 128 : 64;
        pcg.mg_doubles = mg_work_doubles(ncap, pcg.mg_cap);
    }
    // e[0] = max_i |m_i - t_i| / t_i, e[1] = min_i m_i, e[2] = sum_i (m_i - t_i)^2 (sorted order)
    void mass_stats(const double *m, double e[3]) {
        mass_errors(m, t_sorted, n, red, red + 3 * PCG_BLOCKS, stream);
        SDOT_CUDA(cudaMemcpyAsync(e, red + 3 * PCG_BLOCKS, 3 * sizeof(double), cudaMemcpyDeviceToHost, stream));
        SDOT_CUDA(cudaStreamSynchronize(stream));
    }
    void set_device_weights_changed() {
        w_dirty = true;
        mark_dirty();
    }

    int solve(const double *target, int mem_space, const sdot_newton_opts &o, sdot_newton_report &rep) {
        const auto t_start = std::chrono::steady_clock::now();
        rep = sdot_newton_report{};
        if (n == 0) throw BadArg("no Diracs: call sdot_set_diracs first");
        if (!target) throw BadArg("null target masses");
        if (o.max_iter < 0 || o.pcg_max_iter <= 0 || !(o.rel_mass_tol >= 0) || !(o.pcg_rel_tol > 0))
            throw BadArg("bad Newton options");
        reserve_newton();
        upload_target(target, mem_space);
        int st = evaluate();
        ++rep.evaluations;
        if (st != SDOT_OK) return st;
        // targets in sorted (tree) order; the order is fixed while the positions are
        gather_sorted(t_orig, perm(), t_sorted, n, stream);
        double et[3];
        mass_stats(t_sorted, et);  // et[1] = min target
        if (!(et[1] > 0)) throw BadArg("target masses must be positive");
        // gauge fix on the row of Dirac 0 (.tcc:62-63), only without ball cut
        long long gauge = -1;
        if (!ball) {
            int g = 0;
            SDOT_CUDA(cudaMemcpyAsync(&g, perm_inv(), sizeof(int), cudaMemcpyDeviceToHost, stream));
            SDOT_CUDA(cudaStreamSynchronize(stream));
            gauge = g;
        }
        SDOT_CUDA(cudaMemcpyAsync(w_old, d_w, size_t(n) * sizeof(double), cudaMemcpyDeviceToDevice, stream));
        double e[3];
        mass_stats(s_mass, e);
        if (o.damping && !(e[1] > 0)) {
            last_error = "a cell is empty at the start weights (damped Newton keeps every cell non-empty)";
            return SDOT_VOID_CELL;
        }
        const double eps0 = 0.5 * std::min(et[1], e[1]);
        double tau_last = 1.0;
        int status = SDOT_NOT_CONVERGED;
        for (int it = 0;; ++it) {
            rep.max_rel_mass_error = e[0];
            rep.min_mass = e[1];
            if (o.verbosity > 0)
                fprintf(stderr, "sdot newton %d: max rel mass error %.3e, min mass %.3e\n", it, e[0], e[1]);
            if (e[0] <= o.rel_mass_tol) {
                status = SDOT_OK;
                break;
            }
            if (it >= o.max_iter) break;
            rep.iterations = it + 1;
            if (!o.damping && !(e[1] > 0)) {
                // reference back-off on an empty cell: w = 0.9 w_old + 0.1 w (.tcc:72-79)
                axpby(w_old, d_w, d_w, 0.9, 0.1, n, stream);
                set_device_weights_changed();
                st = evaluate();
                ++rep.evaluations;
                if (st != SDOT_OK) return st;
                mass_stats(s_mass, e);
                continue;
            }
            SDOT_CUDA(cudaMemcpyAsync(w_old, d_w, size_t(n) * sizeof(double), cudaMemcpyDeviceToDevice, stream));
            axpby(s_mass, t_sorted, rhs, 1.0, -1.0, n, stream);  // v_values -= masses (.tcc:89-90)
            PcgResult pr;
            if (o.pcg_fp32) {
                reserve_fp32();
                rows_to_float(rows, n, val32, side32, stream);
                pr = pcg_solve_refined(rows, val32, side32, n, gauge, rhs, dir, o.pcg_rel_tol, o.pcg_max_iter, pcg,
                                       pcg32, ref_buf, stream, 1e-4, 32, o.preconditioner == 0);
            } else {
                pr = pcg_solve(rows, n, gauge, rhs, dir, o.pcg_rel_tol, o.pcg_max_iter, pcg, stream, 32,
                               stream != nullptr, o.preconditioner == 0);
            }
            rep.pcg_iterations += pr.iterations;
            rep.pcg_levels = pr.levels;
            if (o.verbosity > 0)
                fprintf(stderr, "sdot newton %d: pcg %d iterations, relative residual %.3e\n", it, pr.iterations,
                        pr.rel_residual);
            // the search starts from 4x the last accepted step length (not
            // from 1): far from the solution, full steps give huge cells
            // whose evaluation is slow or overflows; near it tau returns to 1
            double tau = std::min(1.0, 4.0 * tau_last), en[3];
            bool accepted = false;
            for (int k = 0; k <= 40; ++k) {
                apply_step(w_old, dir, perm(), tau, d_w, n, stream);  // weights -= dw (.tcc:106-109)
                set_device_weights_changed();
                st = evaluate();
                ++rep.evaluations;
                if (st == SDOT_CAPACITY && o.damping) {
                    // a trial step so long that a cell outgrew the kernels'
                    // polyhedra is rejected like one that raised the error
                    tau *= 0.5;
                    continue;
                }
                if (st != SDOT_OK) return st;
                mass_stats(s_mass, en);
                if (!o.damping || en[0] <= o.rel_mass_tol ||
                    (en[1] >= eps0 && std::sqrt(en[2]) <= (1.0 - 0.5 * tau) * std::sqrt(e[2]))) {
                    accepted = true;
                    tau_last = tau;
                    break;
                }
                tau *= 0.5;
            }
            if (!accepted) {
                // no acceptable step: keep the last accepted weights (and
                // their cells, so that the outputs match the weights)
                SDOT_CUDA(cudaMemcpyAsync(d_w, w_old, size_t(n) * sizeof(double), cudaMemcpyDeviceToDevice, stream));
                set_device_weights_changed();
                st = evaluate();
                ++rep.evaluations;
                if (st != SDOT_OK) return st;
                char buf[160];
                snprintf(buf, sizeof buf,
                         "damped Newton: no step length decreased the mass error (max relative mass error %.3e)", e[0]);
                last_error = buf;
                break;
            }
            e[0] = en[0];
            e[1] = en[1];
            e[2] = en[2];
        }
        rep.time_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
        if (status == SDOT_NOT_CONVERGED && last_error.empty()) last_error = "Newton did not reach the tolerance";
        return status;
    }

    void upload_target(const double *target, int mem_space) {
        SDOT_CUDA(cudaMemcpyAsync(t_orig, target, size_t(n) * sizeof(double),
                                  mem_space == SDOT_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                  stream));
    }
};

namespace {

int fail(sdot_ctx *c, int code, const std::string &msg) {
    if (c) c->last_error = msg;
    return code;
}

template <class F>
int guarded(sdot_ctx *c, const F &f) {
    if (!c) return SDOT_BAD_ARG;
    try {
        cudaSetDevice(c->device);
        return f();
    } catch (const CudaError &e) {
        if (e.err == cudaErrorMemoryAllocation) {
            cudaGetLastError();
            return fail(c, SDOT_OOM, std::string("out of device memory in ") + e.where);
        }
        return fail(c, SDOT_CUDA_ERROR, std::string(cudaGetErrorString(e.err)) + " in " + e.where);
    } catch (const BadArg &e) {
        return fail(c, SDOT_BAD_ARG, e.what());
    } catch (const Unsupported &e) {
        return fail(c, SDOT_UNSUPPORTED, e.what());
    } catch (const std::bad_alloc &) {
        return fail(c, SDOT_OOM, "out of host memory");
    } catch (const std::exception &e) {
        return fail(c, SDOT_CUDA_ERROR, e.what());
    }
}

void upload(double *dst, const double *src, size_t count, int mem_space, cudaStream_t st) {
    SDOT_CUDA(cudaMemcpyAsync(dst, src, count * sizeof(double),
                              mem_space == SDOT_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
}

}  // namespace

extern "C" {

sdot_ctx *sdot_create(int dim, int precision, const sdot_options *opt) {
    if (dim != 2 && dim != 3) return nullptr;
    if (precision != SDOT_FP64 && precision != SDOT_MIXED) return nullptr;
    sdot_ctx *c = nullptr;
    try {
        c = new sdot_ctx();
    } catch (...) {
        return nullptr;
    }
    c->dim = dim;
    c->precision = precision;
    int dev = 0;
    cudaGetDevice(&dev);
    if (opt && opt->device >= 0) dev = opt->device;
    c->device = dev;
    if (opt && opt->max_diracs_per_cell > 0) c->max_per_leaf = opt->max_diracs_per_cell;
    if (cudaSetDevice(dev) != cudaSuccess) {
        delete c;
        return nullptr;
    }
    if (opt && opt->stream) {
        c->stream = static_cast<cudaStream_t>(opt->stream);
    } else {
        if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
            delete c;
            return nullptr;
        }
        c->own_stream = true;
    }
    return c;
}

void sdot_destroy(sdot_ctx *ctx) { delete ctx; }

const char *sdot_last_error(const sdot_ctx *ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }

int sdot_set_stream(sdot_ctx *ctx, void *stream) {
    return guarded(ctx, [&] {
        SDOT_CUDA(cudaStreamSynchronize(ctx->stream));
        if (stream) {
            if (ctx->own_stream) SDOT_CUDA(cudaStreamDestroy(ctx->stream));
            ctx->own_stream = false;
            ctx->stream = static_cast<cudaStream_t>(stream);
        } else if (!ctx->own_stream) {
            cudaStream_t s = nullptr;
            SDOT_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
            ctx->stream = s;
            ctx->own_stream = true;
        }
        return int(SDOT_OK);
    });
}

int sdot_set_diracs(sdot_ctx *ctx, const double *positions, const double *weights, int64_t n, int mem_space) {
    return guarded(ctx, [&] {
        if (n < 0 || (n > 0 && (!positions || !weights))) throw BadArg("bad Dirac arrays");
        if (n >= (1LL << 31) - 1) throw BadArg("at most 2^31 - 2 Diracs per context");
        if (n > ctx->cap) {
            dalloc(ctx->d_pos, size_t(ctx->dim) * n);
            dalloc(ctx->d_w, size_t(n));
            ctx->cap = n;
        }
        ctx->n = n;
        if (n) {
            upload(ctx->d_pos, positions, size_t(ctx->dim) * n, mem_space, ctx->stream);
            upload(ctx->d_w, weights, size_t(n), mem_space, ctx->stream);
        }
        ctx->pos_dirty = ctx->w_dirty = true;
        ctx->mark_dirty();
        return int(SDOT_OK);
    });
}

int sdot_set_weights(sdot_ctx *ctx, const double *weights, int mem_space) {
    return guarded(ctx, [&] {
        if (!weights && ctx->n) throw BadArg("null weights");
        if (ctx->n) upload(ctx->d_w, weights, size_t(ctx->n), mem_space, ctx->stream);
        ctx->w_dirty = true;
        ctx->mark_dirty();
        return int(SDOT_OK);
    });
}

int sdot_add_box_shape(sdot_ctx *ctx, const double *p0, const double *p1, double coeff) {
    return guarded(ctx, [&] {
        if (!p0 || !p1) throw BadArg("null box corner");
        ctx->has_image = false;
        if (ctx->dim == 3) {
            sdot_ctx::Item3 b{{p0[0], p0[1], p0[2]}, {p1[0], p1[1], p1[2]}, coeff, {}};
            ctx->items3.push_back(b);
            ctx->planes3_dirty = true;
        } else {
            ctx->items.push_back(box_item(p0[0], p0[1], p1[0], p1[1], coeff));
        }
        ctx->dom_dirty = true;
        ctx->mark_dirty();
        return int(SDOT_OK);
    });
}

int sdot_add_convex_polyhedron_shape(sdot_ctx *ctx, const double *points, const double *normals, int64_t m,
                                     double coeff) {
    return guarded(ctx, [&] {
        if (m <= 0 || !points || !normals) throw BadArg("bad convex polyhedron");
        if (ctx->dim == 3) {
            // ConvexPolyhedronAssembly::add_convex_polyhedron (.tcc:7-33): the
            // bounding box of the points inflated by its size on each side,
            // cut by each (point, normalized normal) half-space
            sdot_ctx::Item3 it;
            it.coeff = coeff;
            for (int d = 0; d < 3; ++d) {
                double mn = std::numeric_limits<double>::max(), mx = -std::numeric_limits<double>::max();
                for (int64_t i = 0; i < m; ++i) {
                    mn = std::min(mn, points[3 * i + d]);
                    mx = std::max(mx, points[3 * i + d]);
                }
                it.lo[d] = mn - (mx - mn);
                it.hi[d] = mx + (mx - mn);
            }
            for (int64_t i = 0; i < m; ++i) {
                const double *q = normals + 3 * i, *p = points + 3 * i;
                const double l = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]) + 1e-40;  // Point3 normalized()
                const double a[3] = {q[0] / l, q[1] / l, q[2] / l};
                it.planes.insert(it.planes.end(), {a[0], a[1], a[2], a[0] * p[0] + a[1] * p[1] + a[2] * p[2]});
            }
            if (it.planes.size() / 4 > 64) throw Unsupported("a 3D shape has more than 64 faces");
            ctx->has_image = false;
            ctx->items3.push_back(std::move(it));
            ctx->planes3_dirty = true;
            ctx->dom_dirty = true;
            ctx->mark_dirty();
            return int(SDOT_OK);
        }
        // ConvexPolyhedronAssembly::add_convex_polyhedron: the bounding box of
        // the points inflated by its size, cut by each (point, normal) half-plane.
        double mn[2], mx[2];
        for (int d = 0; d < 2; ++d) {
            mn[d] = std::numeric_limits<double>::max();
            mx[d] = -std::numeric_limits<double>::max();
            for (int64_t i = 0; i < m; ++i) {
                mn[d] = std::min(mn[d], points[2 * i + d]);
                mx[d] = std::max(mx[d], points[2 * i + d]);
            }
        }
        double dx = mx[0] - mn[0], dy = mx[1] - mn[1];
        const int cap = int(4 + m + 2);
        HostPoly hp(cap);
        double bx[4] = {mn[0] - dx, mx[0] + dx, mx[0] + dx, mn[0] - dx};
        double by[4] = {mn[1] - dy, mn[1] - dy, mx[1] + dy, mx[1] + dy};
        for (int k = 0; k < 4; ++k) {
            hp.x[k] = bx[k];
            hp.y[k] = by[k];
            hp.id[k] = -1 - k;
        }
        int nv = 4;
        std::vector<double> un(2 * m);
        for (int64_t i = 0; i < m; ++i) {
            // Point2 normalized(): p / (|p| + 1e-40)
            double nx = normals[2 * i], ny = normals[2 * i + 1];
            double d = std::sqrt(nx * nx + ny * ny) + 1e-40;
            un[2 * i] = nx / d;
            un[2 * i + 1] = ny / d;
            nv = plane_cut(hp.view(), nv, cap, points[2 * i], points[2 * i + 1], un[2 * i], un[2 * i + 1], int(i));
            if (nv <= 0) break;
        }
        if (nv <= 0) throw BadArg("empty convex polyhedron");
        Item2 it;
        it.coeff = coeff;
        for (int k = 0; k < nv; ++k) {
            it.xy.push_back(hp.x[k]);
            it.xy.push_back(hp.y[k]);
            int id = hp.id[k];
            if (id >= 0) {
                it.nrm.push_back(un[2 * id]);
                it.nrm.push_back(un[2 * id + 1]);
            } else {
                it.nrm.push_back(kBoxNrm[-1 - id][0]);
                it.nrm.push_back(kBoxNrm[-1 - id][1]);
            }
        }
        ctx->has_image = false;
        ctx->items.push_back(std::move(it));
        ctx->dom_dirty = true;
        ctx->mark_dirty();
        return int(SDOT_OK);
    });
}

int sdot_add_simplex_shape(sdot_ctx *ctx, const double *pts, double coeff) {
    return guarded(ctx, [&] {
        if (!pts) throw BadArg("null simplex");
        if (ctx->dim == 3) {
            // a tetrahedron: its bounding box cut by its four face planes, each
            // oriented away from the opposite vertex
            sdot_ctx::Item3 it;
            it.coeff = coeff;
            for (int d = 0; d < 3; ++d) {
                it.lo[d] = std::min(std::min(pts[d], pts[3 + d]), std::min(pts[6 + d], pts[9 + d]));
                it.hi[d] = std::max(std::max(pts[d], pts[3 + d]), std::max(pts[6 + d], pts[9 + d]));
            }
            const int face[4][4] = {{1, 2, 3, 0}, {0, 2, 3, 1}, {0, 1, 3, 2}, {0, 1, 2, 3}};  // 3 vertices, opposite
            for (const auto &f : face) {
                const double *a = pts + 3 * f[0], *b = pts + 3 * f[1], *c = pts + 3 * f[2], *o = pts + 3 * f[3];
                const double u[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]}, v[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
                double nrm[3] = {u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]};
                const double l = std::sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2]);
                if (!(l > 0)) throw BadArg("degenerate simplex");
                double side = nrm[0] * (o[0] - a[0]) + nrm[1] * (o[1] - a[1]) + nrm[2] * (o[2] - a[2]);
                const double sg = side > 0 ? -1.0 : 1.0;
                for (double &x : nrm) x *= sg / l;
                it.planes.insert(it.planes.end(), {nrm[0], nrm[1], nrm[2], nrm[0] * a[0] + nrm[1] * a[1] + nrm[2] * a[2]});
            }
            ctx->has_image = false;
            ctx->items3.push_back(std::move(it));
            ctx->planes3_dirty = true;
            ctx->dom_dirty = true;
            ctx->mark_dirty();
            return int(SDOT_OK);
        }
        // ConvexPolyhedron2( Simplex ) (ConvexPolyhedron2.tcc:19-60)
        double p[3][2] = {{pts[0], pts[1]}, {pts[2], pts[3]}, {pts[4], pts[5]}};
        double cx = 1.0 / 3 * (p[0][0] + p[1][0] + p[2][0]), cy = 1.0 / 3 * (p[0][1] + p[1][1] + p[2][1]);
        auto nrm = [](const double *a, const double *b, double *o) {
            double vx = a[0] - b[0], vy = a[1] - b[1];
            double rx = -vy, ry = vx;  // rot90
            double l = std::sqrt(rx * rx + ry * ry);
            o[0] = rx / l;
            o[1] = ry / l;
        };
        double n0[2], n1[2], n2[2];
        nrm(p[0], p[1], n0);
        nrm(p[1], p[2], n1);
        nrm(p[2], p[0], n2);
        Item2 it;
        it.coeff = coeff;
        if ((p[0][0] - cx) * n0[0] + (p[0][1] - cy) * n0[1] < 0) {
            it.xy = {p[0][0], p[0][1], p[2][0], p[2][1], p[1][0], p[1][1]};
            it.nrm = {-n2[0], -n2[1], -n1[0], -n1[1], -n0[0], -n0[1]};
        } else {
            it.xy = {p[0][0], p[0][1], p[1][0], p[1][1], p[2][0], p[2][1]};
            it.nrm = {n0[0], n0[1], n1[0], n1[1], n2[0], n2[1]};
        }
        ctx->has_image = false;
        ctx->items.push_back(std::move(it));
        ctx->dom_dirty = true;
        ctx->mark_dirty();
        return int(SDOT_OK);
    });
}

int sdot_set_image_density(sdot_ctx *ctx, const double *min_pt, const double *max_pt, const double *data,
                           const int64_t *sizes, int nb_coeffs) {
    return guarded(ctx, [&] {
        if (!min_pt || !max_pt || !data || !sizes) throw BadArg("null image argument");
        if (nb_coeffs != 1 && !(nb_coeffs == 6 && ctx->dim == 2))
            throw Unsupported("images have nb_coeffs = 1 (piecewise constant), or 6 (piecewise quadratic) in 2D "
                              "(Polynomial.h:53-58)");
        long long np = 1;
        for (int d = 0; d < ctx->dim; ++d) {
            if (sizes[d] <= 0 || sizes[d] > (1 << 30)) throw BadArg("bad image size");
            np *= sizes[d];
        }
        ctx->items.clear();
        ctx->has_image = true;
        for (int d = 0; d < 3; ++d) {
            ctx->img_lo[d] = d < ctx->dim ? min_pt[d] : 0.0;
            ctx->img_hi[d] = d < ctx->dim ? max_pt[d] : 1.0;
            ctx->img_size[d] = d < ctx->dim ? sizes[d] : 1;
        }
        ctx->img_ncoeffs = nb_coeffs;
        ctx->img_data.assign(data, data + np * nb_coeffs);
        ctx->dom_dirty = true;
        ctx->mark_dirty();
        return int(SDOT_OK);
    });
}

int sdot_set_polynomial_density(sdot_ctx *ctx, const double *coeffs, int nb_coeffs) {
    return guarded(ctx, [&] {
        if (!coeffs) throw BadArg("null coefficients");
        if (ctx->dim != 3) throw Unsupported("polynomial densities are available in 3D only");
        if (nb_coeffs != 1 && nb_coeffs != 8) throw BadArg("nb_coeffs must be 1 or 8");
        for (int k = 0; k < nb_coeffs; ++k)
            if (!std::isfinite(coeffs[k])) throw BadArg("non-finite density coefficient");
        for (int k = 0; k < 8; ++k) ctx->poly3[k] = k < nb_coeffs ? coeffs[k] : 0.0;
        ctx->has_poly = nb_coeffs == 8;
        ctx->dom_dirty = true;
        ctx->mark_dirty();
        return int(SDOT_OK);
    });
}

int sdot_clear_domain(sdot_ctx *ctx) {
    return guarded(ctx, [&] {
        ctx->items.clear();
        ctx->items3.clear();
        ctx->planes3_dirty = true;
        ctx->has_poly = false;
        for (int k = 0; k < 8; ++k) ctx->poly3[k] = k == 0 ? 1.0 : 0.0;
        ctx->has_image = false;
        ctx->dom_dirty = true;
        ctx->mark_dirty();
        return int(SDOT_OK);
    });
}

static double domain_measure(const sdot_ctx *ctx) {
    if (ctx->has_image) {
        // ScaledImage::measure (ScaledImage.tcc:36-69): the mean over the
        // pixels of the density's average on the pixel, times the area
        const long long nx = ctx->img_size[0], ny = ctx->img_size[1], np = nx * ny * ctx->img_size[2];
        double s = 0;
        if (ctx->img_ncoeffs == 6) {
            // average of c0 + c1 x + c2 y + c3 x^2 + c4 xy + c5 y^2 on a pixel
            // of centre (cx, cy) and size dx x dy: the value at the centre
            // plus (c3 dx^2 + c5 dy^2) / 12
            const double dx = (ctx->img_hi[0] - ctx->img_lo[0]) / double(nx);
            const double dy = (ctx->img_hi[1] - ctx->img_lo[1]) / double(ny);
            const double *c = ctx->img_data.data();
            for (long long yi = 0, o = 0; yi < ny; ++yi)
                for (long long xi = 0; xi < nx; ++xi, ++o) {
                    const double cx = ctx->img_lo[0] + dx * double(xi) + 0.5 * dx;
                    const double cy = ctx->img_lo[1] + dy * double(yi) + 0.5 * dy;
                    s += c[o] + c[np + o] * cx + c[2 * np + o] * cy + c[3 * np + o] * cx * cx +
                         c[4 * np + o] * cx * cy + c[5 * np + o] * cy * cy +
                         (1.0 / 12.0) * (c[3 * np + o] * dx * dx + c[5 * np + o] * dy * dy);
                }
        } else {
            for (double v : ctx->img_data) s += v;
        }
        s /= double(np);
        for (int d = 0; d < ctx->dim; ++d) s *= ctx->img_hi[d] - ctx->img_lo[d];
        return s;
    }
    double res = 0;
    for (const Item2 &it : ctx->items) res += it.coeff * it.area();
    for (const sdot_ctx::Item3 &b : ctx->items3) {
        double f = 0;
        if (b.planes.empty()) {
            // integral over the box of the multilinear factor: per monomial, a
            // product over the axes of (hi - lo) or (hi^2 - lo^2) / 2
            static const int axes[8] = {0, 1, 2, 4, 3, 5, 6, 7};  // bit d: u_d in the monomial
            for (int k = 0; k < 8; ++k) {
                double t = ctx->poly3[k];
                for (int d = 0; d < 3; ++d)
                    t *= (axes[k] >> d & 1) ? 0.5 * (b.hi[d] * b.hi[d] - b.lo[d] * b.lo[d]) : b.hi[d] - b.lo[d];
                f += t;
            }
        } else {
            // the shape's polyhedron built on the host and integrated
            // (ConvexPolyhedron3::measure with the multilinear factor)
            HostPoly3 hp = HostPoly3::box(b.lo, b.hi);
            for (size_t k = 0; k + 3 < b.planes.size(); k += 4) hp.cut(&b.planes[k], b.planes[k + 3]);
            f = hp.integrate(ctx->poly3);
        }
        res += b.coeff * f;
    }
    return res;
}

int sdot_normalize_domain(sdot_ctx *ctx) {
    return guarded(ctx, [&] {
        double mea = domain_measure(ctx);
        if (mea != 0) {
            if (ctx->has_image)
                for (double &v : ctx->img_data) v /= mea;
            else {
                for (Item2 &it : ctx->items) it.coeff /= mea;
                for (sdot_ctx::Item3 &b : ctx->items3) b.coeff /= mea;
            }
        }
        ctx->dom_dirty = true;
        ctx->mark_dirty();
        return int(SDOT_OK);
    });
}

int sdot_domain_measure(sdot_ctx *ctx, double *measure) {
    return guarded(ctx, [&] {
        if (!measure) throw BadArg("null output");
        *measure = domain_measure(ctx);
        return int(SDOT_OK);
    });
}

int sdot_set_translations(sdot_ctx *ctx, const double *translations, int64_t count) {
    return guarded(ctx, [&] {
        if (count < 0 || (count > 0 && !translations)) throw BadArg("bad translations");
        if (ctx->dim != 2 && count > 0) throw Unsupported("periodic translations are available in 2D only");
        if (count > 64) throw BadArg("at most 64 translations");
        ctx->trans_h.assign(translations, translations + 2 * count);
        if (count) {
            dalloc(ctx->d_trans, size_t(2 * count));
            SDOT_CUDA(cudaMemcpy(ctx->d_trans, ctx->trans_h.data(), size_t(2 * count) * sizeof(double),
                                 cudaMemcpyHostToDevice));
        }
        ctx->dom_dirty = true;
        ctx->mark_dirty();
        return int(SDOT_OK);
    });
}

int sdot_set_ball_cut(sdot_ctx *ctx, int on) {
    return guarded(ctx, [&] {
        ctx->ball = on ? 1 : 0;
        ctx->mark_dirty();
        return int(SDOT_OK);
    });
}

int sdot_evaluate(sdot_ctx *ctx) {
    return guarded(ctx, [&] { return ctx->evaluate(); });
}

int sdot_get_integrals(sdot_ctx *ctx, double *out, int mem_space) {
    return guarded(ctx, [&] {
        if (!out) throw BadArg("null output");
        int st = ctx->evaluate();
        ctx->copy_out(out, ctx->o_mass, size_t(ctx->n) * sizeof(double), mem_space);
        SDOT_CUDA(cudaStreamSynchronize(ctx->stream));
        return st;
    });
}

int sdot_get_centroids(sdot_ctx *ctx, double *out_c, double *out_m, int mem_space) {
    return guarded(ctx, [&] {
        if (!out_c) throw BadArg("null output");
        int st = ctx->evaluate();
        ctx->copy_out(out_c, ctx->o_ctd, size_t(ctx->n) * ctx->dim * sizeof(double), mem_space);
        if (out_m) ctx->copy_out(out_m, ctx->o_mass_c, size_t(ctx->n) * sizeof(double), mem_space);
        SDOT_CUDA(cudaStreamSynchronize(ctx->stream));
        return st;
    });
}

int sdot_get_der_integrals_wrt_weights(sdot_ctx *ctx, int64_t *offsets, int64_t *columns, double *values,
                                       double *masses, int64_t *nnz_inout, int stop_if_void, int mem_space) {
    return guarded(ctx, [&] {
        if (!nnz_inout) throw BadArg("null nnz");
        int st = ctx->evaluate();
        if (st != SDOT_OK) return st;
        if (!columns) {
            *nnz_inout = ctx->nnz;
            return int(SDOT_OK);
        }
        if (*nnz_inout < ctx->nnz) throw BadArg("columns/values buffers smaller than nnz");
        if (!offsets || !values || !masses) throw BadArg("null output");
        const long long n = ctx->n, nnz = ctx->nnz;
        long long *dcols = reinterpret_cast<long long *>(columns);
        double *dvals = values;
        if (mem_space != SDOT_DEVICE) {
            // host outputs: written on the device into the context's staging
            // buffers, then copied
            ctx->reserve_stage(nnz);
            dcols = ctx->stage_i;
            dvals = ctx->stage_v;
        }
        csr_write(ctx->rows, n, ctx->perm(), ctx->offsets, dcols, dvals, ctx->stream);
        ctx->copy_out(offsets, ctx->offsets, size_t(n + 1) * sizeof(long long), mem_space);
        ctx->copy_out(masses, ctx->o_mass, size_t(n) * sizeof(double), mem_space);
        if (mem_space != SDOT_DEVICE) {
            SDOT_CUDA(cudaMemcpyAsync(columns, dcols, nnz * sizeof(long long), cudaMemcpyDeviceToHost, ctx->stream));
            SDOT_CUDA(cudaMemcpyAsync(values, dvals, nnz * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        }
        SDOT_CUDA(cudaStreamSynchronize(ctx->stream));
        *nnz_inout = nnz;
        if (stop_if_void && ctx->n_void > 0) {
            // reference: any v == 0 -> 1 (get_der_integrals_wrt_weights.h:93-96);
            // the empty cells were counted on the device by the evaluation
            ctx->last_error = "void cell";
            return int(SDOT_VOID_CELL);
        }
        return int(SDOT_OK);
    });
}

int sdot_get_neighbors(sdot_ctx *ctx, int64_t *offsets, int64_t *ids, int64_t *count_inout, int mem_space) {
    return guarded(ctx, [&] {
        if (!count_inout) throw BadArg("null count");
        ctx->evaluate_neighbors();
        if (!ids) {
            *count_inout = ctx->nb_total;
            return int(SDOT_OK);
        }
        if (*count_inout < ctx->nb_total) throw BadArg("ids buffer smaller than count");
        if (!offsets) throw BadArg("null offsets");
        const long long n = ctx->n, tot = ctx->nb_total;
        long long *dids = reinterpret_cast<long long *>(ids);
        if (mem_space != SDOT_DEVICE) {
            ctx->reserve_stage(tot);
            dids = ctx->stage_i;
        }
        nb_write(ctx->nb, n, ctx->perm(), ctx->nb_offsets, dids, ctx->stream);
        if (mem_space != SDOT_DEVICE)
            SDOT_CUDA(cudaMemcpyAsync(ids, dids, tot * sizeof(long long), cudaMemcpyDeviceToHost, ctx->stream));
        ctx->copy_out(offsets, ctx->nb_offsets, size_t(n + 1) * sizeof(long long), mem_space);
        SDOT_CUDA(cudaStreamSynchronize(ctx->stream));
        *count_inout = tot;
        return int(SDOT_OK);
    });
}

int sdot_get_image_integrals(sdot_ctx *ctx, const double *min_pt, const double *max_pt, const int64_t *nb_pixels,
                             double *out, int mem_space) {
    return guarded(ctx, [&] {
        if (!min_pt || !max_pt || !nb_pixels || !out) throw BadArg("null argument");
        ctx->rasterize(min_pt, max_pt, nb_pixels[0], nb_pixels[1], false);
        ctx->copy_out(out, ctx->ras_buf, size_t(3 * nb_pixels[0] * nb_pixels[1]) * sizeof(double), mem_space);
        SDOT_CUDA(cudaStreamSynchronize(ctx->stream));
        return ctx->finish_status();
    });
}

int sdot_get_image_of_cell_nums(sdot_ctx *ctx, const double *min_pt, const double *max_pt, const int64_t *nb_pixels,
                                int64_t *out, int mem_space) {
    return guarded(ctx, [&] {
        if (!min_pt || !max_pt || !nb_pixels || !out) throw BadArg("null argument");
        ctx->rasterize(min_pt, max_pt, nb_pixels[0], nb_pixels[1], true);
        ctx->copy_out(out, ctx->ras_nums, size_t(nb_pixels[0] * nb_pixels[1]) * sizeof(int64_t), mem_space);
        SDOT_CUDA(cudaStreamSynchronize(ctx->stream));
        return ctx->finish_status();
    });
}

int sdot_get_der_centroids_and_integrals_wrt_weight_and_positions(sdot_ctx *ctx, int64_t *offsets,
                                                                   int64_t *columns, double *values,
                                                                   double *v_values, int64_t *nnz_inout,
                                                                   int mem_space) {
    return guarded(ctx, [&] {
        if (!nnz_inout) throw BadArg("null nnz");
        if (ctx->dim != 2) throw Unsupported("position derivatives are available in 2D");
        ctx->check_domain();
        if (ctx->ball) throw Unsupported("position derivatives with the disc clip are not available in this build");
        if (ctx->mode != DM_SINGLE && ctx->mode != DM_PERIODIC)
            throw Unsupported("position derivatives are available for one-shape domains");
        ctx->evaluate_neighbors();
        const long long n = ctx->n;
        // block counts per Dirac, their scan, then the rows
        ctx->reserve_stage(std::max<long long>(n + 1, 1));
        long long *counts = ctx->cnt_orig, *boff = ctx->stage_i;
        SDOT_CUDA(cudaMemsetAsync(ctx->err, 0, sizeof(unsigned), ctx->stream));
        derpos_count(ctx->nb, n, ctx->tree2.pos, ctx->tree2.w, ctx->perm(), ctx->start_n, ctx->d_start, ctx->coeff,
                     int(ctx->trans_h.size() / 2), ctx->d_trans, counts, ctx->err, ctx->stream);
        scan_exclusive_total<long long>(counts, boff, n, ctx->scan_tmp, ctx->stream);
        long long total = 0;
        unsigned e = 0;
        SDOT_CUDA(cudaMemcpyAsync(&total, boff + n, sizeof(long long), cudaMemcpyDeviceToHost, ctx->stream));
        SDOT_CUDA(cudaMemcpyAsync(&e, ctx->err, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream));
        SDOT_CUDA(cudaStreamSynchronize(ctx->stream));
        if (e & DE_CAPACITY) {
            ctx->last_error = "a cell has more than 64 vertices (the position derivatives' capacity)";
            return int(SDOT_CAPACITY);
        }
        const long long nnz = 9 * total;
        if (!columns) {
            *nnz_inout = nnz;
            return ctx->finish_status();
        }
        if (*nnz_inout < nnz) throw BadArg("columns/values buffers smaller than nnz");
        if (!offsets || !values || !v_values) throw BadArg("null output");
        long long *d_off = reinterpret_cast<long long *>(offsets), *d_col = reinterpret_cast<long long *>(columns);
        double *d_val = values, *d_v = v_values;
        if (mem_space != SDOT_DEVICE) {
            ctx->reserve_derpos(n, nnz);
            d_off = ctx->dp_off;
            d_col = ctx->dp_col;
            d_val = ctx->dp_val;
            d_v = ctx->dp_v;
        }
        derpos_write(ctx->nb, n, ctx->tree2.pos, ctx->tree2.w, ctx->perm(), ctx->start_n, ctx->d_start, ctx->coeff,
                     int(ctx->trans_h.size() / 2), ctx->d_trans, boff, d_off, d_col, d_val, d_v, ctx->stream);
        if (mem_space != SDOT_DEVICE) {
            SDOT_CUDA(cudaMemcpyAsync(offsets, d_off, size_t(3 * n + 1) * sizeof(long long), cudaMemcpyDeviceToHost,
                                      ctx->stream));
            SDOT_CUDA(cudaMemcpyAsync(columns, d_col, size_t(nnz) * sizeof(long long), cudaMemcpyDeviceToHost, ctx->stream));
            SDOT_CUDA(cudaMemcpyAsync(values, d_val, size_t(nnz) * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
            SDOT_CUDA(cudaMemcpyAsync(v_values, d_v, size_t(3 * n) * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        }
        SDOT_CUDA(cudaStreamSynchronize(ctx->stream));
        *nnz_inout = nnz;
        return ctx->finish_status();
    });
}

int sdot_solve(sdot_ctx *ctx, const double *target, int mem_space, const sdot_newton_opts *opts,
               sdot_newton_report *report) {
    return guarded(ctx, [&] {
        sdot_newton_opts o{150, 1e-10, 20000, 1e-12, 1, 0, 0, 0};
        if (opts) o = *opts;
        sdot_newton_report r{};
        ctx->last_error.clear();
        const int st = ctx->solve(target, mem_space, o, r);
        if (report) *report = r;
        return st;
    });
}

int sdot_csr_solve(const int64_t *offsets, const int64_t *columns, const double *values, int64_t n, const double *b,
                   double *x, int gauge_fix, double rel_tol, int max_iter, int mem_space, int64_t *iterations,
                   double *rel_residual, char *errbuf, int64_t errbuf_len) {
    auto err = [&](int code, const std::string &msg) {
        if (errbuf && errbuf_len > 0) {
            const size_t k = std::min<size_t>(msg.size(), size_t(errbuf_len - 1));
            std::memcpy(errbuf, msg.data(), k);
            errbuf[k] = 0;
        }
        return code;
    };
    if (n < 0 || (n > 0 && (!offsets || !columns || !values || !b || !x)) || max_iter <= 0 || !(rel_tol > 0))
        return err(SDOT_BAD_ARG, "bad CSR solve arguments");
    if (errbuf && errbuf_len > 0) errbuf[0] = 0;
    if (n == 0) return SDOT_OK;
    cudaStream_t st = nullptr;
    long long *d_off = nullptr, *d_col = nullptr;
    double *d_val = nullptr, *d_b = nullptr, *d_x = nullptr, *work = nullptr;
    auto release = [&] {
        if (mem_space != SDOT_DEVICE) {
            dfree(d_off); dfree(d_col); dfree(d_val); dfree(d_b); dfree(d_x);
        }
        dfree(work);
        if (st) cudaStreamDestroy(st);
    };
    try {
        SDOT_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        long long nnz = 0;
        if (mem_space == SDOT_DEVICE) {
            SDOT_CUDA(cudaMemcpyAsync(&nnz, offsets + n, sizeof(long long), cudaMemcpyDeviceToHost, st));
            SDOT_CUDA(cudaStreamSynchronize(st));
            d_off = (long long *)offsets;
            d_col = (long long *)columns;
            d_val = (double *)values;
            d_b = (double *)b;
            d_x = x;
        } else {
            nnz = offsets[n];
            dalloc(d_off, size_t(n) + 1);
            dalloc(d_col, size_t(nnz));
            dalloc(d_val, size_t(nnz));
            dalloc(d_b, size_t(n));
            dalloc(d_x, size_t(n));
            SDOT_CUDA(cudaMemcpyAsync(d_off, offsets, (n + 1) * sizeof(long long), cudaMemcpyHostToDevice, st));
            SDOT_CUDA(cudaMemcpyAsync(d_col, columns, nnz * sizeof(long long), cudaMemcpyHostToDevice, st));
            SDOT_CUDA(cudaMemcpyAsync(d_val, values, nnz * sizeof(double), cudaMemcpyHostToDevice, st));
            SDOT_CUDA(cudaMemcpyAsync(d_b, b, n * sizeof(double), cudaMemcpyHostToDevice, st));
        }
        dalloc(work, pcg_work_doubles(n));
        PcgWork w;
        pcg_bind(w, work, n);
        const PcgResult r = pcg_solve_csr(CsrMat{d_off, d_col, d_val}, n, gauge_fix ? 0 : -1, d_b, d_x, rel_tol,
                                          max_iter, w, st);
        if (mem_space != SDOT_DEVICE)
            SDOT_CUDA(cudaMemcpyAsync(x, d_x, n * sizeof(double), cudaMemcpyDeviceToHost, st));
        SDOT_CUDA(cudaStreamSynchronize(st));
        if (iterations) *iterations = r.iterations;
        if (rel_residual) *rel_residual = r.rel_residual;
        release();
        return r.converged ? int(SDOT_OK) : err(SDOT_NOT_CONVERGED, "conjugate gradients did not reach the tolerance");
    } catch (const CudaError &e) {
        release();
        return err(e.err == cudaErrorMemoryAllocation ? SDOT_OOM : SDOT_CUDA_ERROR,
                   std::string(cudaGetErrorString(e.err)) + " in " + e.where);
    }
}

int sdot_get_weights(sdot_ctx *ctx, double *out, int mem_space) {
    return guarded(ctx, [&] {
        if (!out) throw BadArg("null output");
        if (ctx->n) ctx->copy_out(out, ctx->d_w, size_t(ctx->n) * sizeof(double), mem_space);
        SDOT_CUDA(cudaStreamSynchronize(ctx->stream));
        return int(SDOT_OK);
    });
}

int sdot_last_timings(const sdot_ctx *ctx, double *t3) {
    if (!ctx || !t3) return SDOT_BAD_ARG;
    for (int k = 0; k < 3; ++k) t3[k] = ctx->times[k];
    return SDOT_OK;
}

int sdot_debug_checks(uint64_t *out6) {
    if (!out6) return SDOT_BAD_ARG;
    unsigned long long a[3], b[3];
    try {
        cells2d_read_checks(a);
        csr_read_checks(b);
    } catch (const CudaError &) {
        return SDOT_CUDA_ERROR;
    }
    for (int k = 0; k < 3; ++k) {
        out6[k] = a[k];
        out6[3 + k] = b[k];
    }
    return SDOT_OK;
}

int sdot_debug_work_counts(uint64_t *out8, int reset) {
    if (!out8) return SDOT_BAD_ARG;
    unsigned long long a[8];
    try {
        cells2d_read_work(a, reset != 0);
    } catch (const CudaError &) {
        return SDOT_CUDA_ERROR;
    }
    for (int k = 0; k < 8; ++k) out8[k] = a[k];
    return SDOT_OK;
}

int sdot_kernel_launches(uint64_t *count) {
    if (!count) return SDOT_BAD_ARG;
    *count = g_launches.load();
    return SDOT_OK;
}

int sdot_last_overflow_count(const sdot_ctx *ctx, int64_t *count) {
    if (!ctx || !count) return SDOT_BAD_ARG;
    *count = ctx->last_ovf;
    return SDOT_OK;
}

}  // extern "C"
