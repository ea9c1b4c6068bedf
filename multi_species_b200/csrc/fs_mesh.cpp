// Host construction of the uniform periodic phase-space panel mesh.
//
// The point ORDER and the panel/neighbour records must be the reference's
// exactly, because point indices are the simulation's data layout and the
// diagnostic files (leaf_point_inds_*) are written in it.  The refinement
// rules follow create_prerefined_mesh (src/structure_files/AMRStructure_amr.cpp:127-230),
// refine_panels (:506-839, 2x2 split) and refine_panels_refine_v (:233-504,
// split in p only), for periodic boundaries and uniform (non-adaptive)
// refinement.  Points are appended in the order the reference allocates their
// indices, so appending immediately gives the same numbering.
//
// The mesh is identical at every remesh of a uniform deck, so it is built once
// per species and cached on the device.
#include <cmath>
#include <functional>

#include "fs_internal.h"

namespace fsb {

namespace {

HostPanel make_panel(int level, int parent, int which, const int* pts, int l, int t, int r, int b,
                     bool lb, bool rb) {
    HostPanel q;
    std::memset(&q, 0, sizeof(q));
    for (int i = 0; i < 9; ++i) q.pts[i] = pts ? pts[i] : -1;
    q.level = level;
    q.parent = parent;
    q.which = which;
    q.child = -1;
    q.left = l;
    q.top = t;
    q.right = r;
    q.bottom = b;
    q.lb = lb;
    q.rb = rb;
    return q;
}

class Refiner {
   public:
    explicit Refiner(HostMesh& m) : m_(m) {}

    int add_point(double x, double p) {
        m_.xs.push_back(x);
        m_.ps.push_back(p);
        return (int)m_.xs.size() - 1;
    }

    // One side of a panel being split 2x2.  Describes which neighbour link is
    // read, which two children of a refined neighbour face this side, which of
    // their points lies on the shared edge, which link of those children points
    // back, and which of our four children (offsets from the first new panel)
    // touch the side.
    struct Side {
        int HostPanel::*nbr;
        int face0, face1;              // neighbour child offsets facing us
        int face_pt;                   // point index (0..8) on the shared edge
        int HostPanel::*back;          // link of the facing children pointing to us
        int own0, own1;                // our children on this side
        bool periodic_copy;            // boundary sides of x get their own points
    };

    // refine_panels: split every flagged panel of the current generation 2x2.
    void split_xp() {
        static const Side kLeft = {&HostPanel::left, 2, 3, 7, &HostPanel::right, 0, 1, true};
        static const Side kBottom = {&HostPanel::bottom, 1, 3, 5, &HostPanel::top, 0, 2, false};
        static const Side kTop = {&HostPanel::top, 0, 2, 3, &HostPanel::bottom, 1, 3, false};
        static const Side kRight = {&HostPanel::right, 0, 1, 1, &HostPanel::left, 2, 3, true};
        const int gen_end = (int)m_.panels.size();
        for (int jj = m_min_; jj < gen_end; ++jj) {
            if (!m_.panels[jj].needs) continue;
            const HostPanel P = m_.panels[jj];
            const double x0 = m_.xs[P.pts[0]], p0 = m_.ps[P.pts[0]];
            const double half_dx = m_.xs[P.pts[3]] - x0, half_dp = m_.ps[P.pts[1]] - p0;
            const double qx = 0.5 * half_dx, qp = 0.5 * half_dp;
            double X[5], Pp[5];
            for (int i = 0; i < 5; ++i) {
                X[i] = x0 + qx * i;
                Pp[i] = p0 + qp * i;
            }
            const int n = (int)m_.panels.size();
            int link[4][4];  // link[child][0=left,1=top,2=right,3=bottom]
            for (auto& c : link)
                for (int& v : c) v = -1;
            // internal links
            link[0][1] = n + 1; link[0][2] = n + 2;
            link[1][2] = n + 3; link[1][3] = n;
            link[2][0] = n;     link[2][1] = n + 3;
            link[3][0] = n + 1; link[3][3] = n + 2;
            int slot_of_side[4] = {0, 3, 1, 2};  // left, bottom, top, right -> link index
            const Side* sides[4] = {&kLeft, &kBottom, &kTop, &kRight};
            const double sx[4][2] = {{X[0], X[0]}, {X[1], X[3]}, {X[1], X[3]}, {X[4], X[4]}};
            const double sp[4][2] = {{Pp[1], Pp[3]}, {Pp[0], Pp[0]}, {Pp[4], Pp[4]}, {Pp[1], Pp[3]}};
            int edge_pt[4][2];
            for (int s = 0; s < 4; ++s) {
                const Side& S = *sides[s];
                const int nb = P.*(S.nbr);
                const int li = slot_of_side[s];
                bool fresh = true;
                if (nb == -2) {
                    link[S.own0][li] = link[S.own1][li] = -2;
                } else if (nb == -1) {
                    HostPanel& pn = m_.panels[m_.panels[P.parent].*(S.nbr)];
                    if (!pn.xp) {
                        pn.needs = 1;
                        need_further = true;
                    }
                } else if (m_.panels[nb].xp) {
                    const int c0 = m_.panels[nb].child + S.face0, c1 = m_.panels[nb].child + S.face1;
                    link[S.own0][li] = c0;
                    link[S.own1][li] = c1;
                    m_.panels[c0].*(S.back) = n + S.own0;
                    m_.panels[c1].*(S.back) = n + S.own1;
                    const bool on_bdry = (s == 0) ? P.lb : (s == 3) ? P.rb : false;
                    if (!(S.periodic_copy && on_bdry)) {
                        edge_pt[s][0] = m_.panels[c0].pts[S.face_pt];
                        edge_pt[s][1] = m_.panels[c1].pts[S.face_pt];
                        fresh = false;
                    }
                } else if (s == 3 && nb == jj) {
                    // a one-panel-wide row is its own right neighbour
                    link[2][2] = n; link[0][0] = n + 2;
                    link[3][2] = n + 1; link[1][0] = n + 3;
                }
                if (fresh) {
                    edge_pt[s][0] = add_point(sx[s][0], sp[s][0]);
                    edge_pt[s][1] = add_point(sx[s][1], sp[s][1]);
                }
            }
            // interior: x1 at p1..p3, x2 at p1,p3, x3 at p1..p3
            const int c12 = add_point(X[1], Pp[1]);
            add_point(X[1], Pp[2]);
            add_point(X[1], Pp[3]);
            const int c16 = add_point(X[2], Pp[1]);
            add_point(X[2], Pp[3]);
            const int c19 = add_point(X[3], Pp[1]);
            add_point(X[3], Pp[2]);
            add_point(X[3], Pp[3]);
            HostPanel& parent = m_.panels[jj];
            parent.xp = 1;
            parent.needs = 0;
            parent.child = n;
            const int* q = P.pts;
            const int e9 = edge_pt[0][0], e10 = edge_pt[0][1], e11 = edge_pt[1][0], e18 = edge_pt[1][1];
            const int e15 = edge_pt[2][0], e22 = edge_pt[2][1], e23 = edge_pt[3][0], e24 = edge_pt[3][1];
            const int pts[4][9] = {
                {q[0], e9, q[1], e11, c12, c12 + 1, q[3], c16, q[4]},
                {q[1], e10, q[2], c12 + 1, c12 + 2, e15, q[4], c16 + 1, q[5]},
                {q[3], c16, q[4], e18, c19, c19 + 1, q[6], e23, q[7]},
                {q[4], c16 + 1, q[5], c19 + 1, c19 + 2, e22, q[7], e24, q[8]}};
            for (int c = 0; c < 4; ++c) {
                const bool lb = (c < 2) ? P.lb : false;
                const bool rb = (c >= 2) ? P.rb : false;
                m_.panels.push_back(make_panel(P.level + 1, jj, c, pts[c], link[c][0], link[c][1],
                                               link[c][2], link[c][3], lb, rb));
            }
        }
    }

    // refine_panels_refine_v: split every flagged panel of the current
    // generation in p only (two children, bottom then top).
    void split_p() {
        const int gen_end = (int)m_.panels.size();
        for (int jj = m_min_; jj < gen_end; ++jj) {
            if (!m_.panels[jj].needs) continue;
            const HostPanel P = m_.panels[jj];
            const double x0 = m_.xs[P.pts[0]], p0 = m_.ps[P.pts[0]];
            const double half_dx = m_.xs[P.pts[3]] - x0, half_dp = m_.ps[P.pts[1]] - p0;
            const double qp = 0.5 * half_dp, qx = 0.5 * half_dx;
            double X[5], Pp[5];
            for (int i = 0; i < 5; ++i) {
                Pp[i] = p0 + qp * i;
                X[i] = x0 + qx * i;
            }
            const int n = (int)m_.panels.size();
            // children links, defaults as in the reference (self links are
            // overwritten when the neighbour is split later in the pass)
            int l0 = n, l1 = n + 1, r0 = n, r1 = n + 1, b0 = -1, t1 = -1;
            auto refined = [&](int i) { return m_.panels[i].xp || m_.panels[i].pr; };
            int e9, e10, e13, e14;
            // left
            bool fresh = true;
            if (P.left == -2) {
                l0 = l1 = -2;
            } else if (P.left == -1) {
                HostPanel& pn = m_.panels[m_.panels[P.parent].left];
                if (!(pn.xp || pn.pr)) pn.needs = 1;
            } else if (refined(P.left)) {
                const HostPanel& L = m_.panels[P.left];
                l0 = L.xp ? L.child + 2 : L.child;
                l1 = L.xp ? L.child + 3 : L.child + 1;
                m_.panels[l0].right = n;
                m_.panels[l1].right = n + 1;
                if (!P.lb) {
                    e9 = m_.panels[l0].pts[7];
                    e10 = m_.panels[l1].pts[7];
                    fresh = false;
                }
            }
            if (fresh) {
                e9 = add_point(X[0], Pp[1]);
                e10 = add_point(X[0], Pp[3]);
            }
            // bottom (no new points on horizontal edges)
            if (P.bottom == -2) {
                b0 = -2;
            } else if (P.bottom >= 0 && !m_.panels[P.bottom].xp) {
                HostPanel& B = m_.panels[P.bottom];
                if (!B.pr) {
                    b0 = P.bottom;
                    B.top = n;
                } else {
                    b0 = B.child + 1;
                    m_.panels[b0].top = n;
                }
            }
            // top
            if (P.top == -2) {
                t1 = -2;
            } else if (P.top >= 0 && !m_.panels[P.top].xp) {
                const HostPanel& T = m_.panels[P.top];
                if (T.pr) {
                    t1 = T.child;
                    m_.panels[t1].bottom = n + 1;
                }
            }
            // right
            fresh = true;
            if (P.right == -2) {
                r0 = r1 = -2;
            } else if (P.right == -1) {
                HostPanel& pn = m_.panels[m_.panels[P.parent].right];
                if (!(pn.xp || pn.pr)) pn.needs = 1;
            } else if (refined(P.right)) {
                r0 = m_.panels[P.right].child;
                r1 = r0 + 1;
                m_.panels[r0].left = n;
                m_.panels[r1].left = n + 1;
                if (!P.rb) {
                    e13 = m_.panels[r0].pts[1];
                    e14 = m_.panels[r1].pts[1];
                    fresh = false;
                }
            }
            if (fresh) {
                e13 = add_point(X[4], Pp[1]);
                e14 = add_point(X[4], Pp[3]);
            }
            const int c11 = add_point(X[2], Pp[1]);
            add_point(X[2], Pp[3]);
            HostPanel& parent = m_.panels[jj];
            parent.pr = 1;
            parent.needs = 0;
            parent.child = n;
            const int* q = P.pts;
            const int a[9] = {q[0], e9, q[1], q[3], c11, q[4], q[6], e13, q[7]};
            const int b[9] = {q[1], e10, q[2], q[4], c11 + 1, q[5], q[7], e14, q[8]};
            m_.panels.push_back(make_panel(P.level + 1, jj, 0, a, l0, n + 1, r0, b0, P.lb, P.rb));
            m_.panels.push_back(make_panel(P.level + 1, jj, 1, b, l1, t1, r1, n, P.lb, P.rb));
        }
    }

    // a coarser neighbour was flagged while splitting (2:1 balance)
    bool need_further = false;

    void flag_generation() {
        for (size_t i = m_min_; i < m_.panels.size(); ++i) m_.panels[i].needs = 1;
    }
    void next_generation(int first) { m_min_ = first; }
    int first() const { return m_min_; }

   private:
    HostMesh& m_;
    int m_min_ = 1;
};

void collect_leaves(const HostMesh& m, int pi, std::vector<int>& out) {
    // iterative DFS with the reference's child order (recursively_set_leaves_weights)
    std::vector<int> stack{pi};
    while (!stack.empty()) {
        int i = stack.back();
        stack.pop_back();
        const HostPanel& P = m.panels[i];
        int nc = P.pr ? 2 : (P.xp ? 4 : 0);
        if (!nc) {
            out.push_back(i);
            continue;
        }
        for (int c = nc - 1; c >= 0; --c) stack.push_back(P.child + c);
    }
}

}  // namespace

void HostMesh::build(int h_, int ph_, double xmin_, double xmax_, double pmin_, double pmax_) {
    if (h_ < 1 || ph_ < 0 || h_ + ph_ > 14) fail(FS_ERR_ARG, "mesh heights out of range");
    h = h_;
    ph = ph_;
    xmin = xmin_;
    xmax = xmax_;
    pmin = pmin_;
    pmax = pmax_;
    panels.clear();
    xs.clear();
    ps.clear();
    leaves.clear();
    const size_t npts = (size_t)(2 * (1 << h) + 1) * (size_t)(2 * (1 << (h + ph)) + 1);
    xs.reserve(npts);
    ps.reserve(npts);
    Refiner R(*this);
    // 25-point root (AMRStructure_amr.cpp:139-195): the 3x3 corner/mid lattice,
    // then the two inner columns, then the right column's odd rows.
    const double dx = (xmax - xmin) / 4, dp = (pmax - pmin) / 4;
    double xi[5], pi[5];
    for (int i = 0; i < 5; ++i) {
        xi[i] = xmin + i * dx;
        pi[i] = pmin + i * dp;
    }
    for (int i = 0; i < 5; i += 2)
        for (int j = 0; j < 5; j += 2) R.add_point(xi[i], pi[j]);
    for (int c = 0; c < 2; ++c) {
        R.add_point(xi[2 * c], pi[1]);
        R.add_point(xi[2 * c], pi[3]);
        for (int j = 0; j < 5; ++j) R.add_point(xi[1 + 2 * c], pi[j]);
    }
    R.add_point(xi[4], pi[1]);
    R.add_point(xi[4], pi[3]);
    const int root_pts[9] = {0, 1, 2, 3, 4, 5, 6, 7, 8};
    panels.push_back(make_panel(0, -1, -1, root_pts, 0, -2, 0, -2, true, true));
    const int c1[9] = {0, 9, 1, 11, 12, 13, 3, 16, 4};
    const int c2[9] = {1, 10, 2, 13, 14, 15, 4, 17, 5};
    const int c3[9] = {3, 16, 4, 18, 19, 20, 6, 23, 7};
    const int c4[9] = {4, 17, 5, 20, 21, 22, 7, 24, 8};
    panels.push_back(make_panel(1, 0, 0, c1, 3, 2, 3, -2, true, false));
    panels.push_back(make_panel(1, 0, 1, c2, 4, -2, 4, 1, true, false));
    panels.push_back(make_panel(1, 0, 2, c3, 1, 4, 1, -2, false, true));
    panels.push_back(make_panel(1, 0, 3, c4, 2, -2, 2, 3, false, true));
    panels[0].xp = 1;
    panels[0].child = 1;
    for (int i = 1; i <= 4; ++i) panels[i].needs = 1;
    R.next_generation(1);
    for (int level = 1; level < h; ++level) {
        const int first = (int)panels.size();
        R.flag_generation();
        R.split_xp();
        R.next_generation(first);
    }
    for (int level = 0; level < ph; ++level) {
        const int first = (int)panels.size();
        R.flag_generation();
        R.split_p();
        R.next_generation(first);
    }
    collect_leaves(*this, 0, leaves);
    if (xs.size() != npts) fail(FS_ERR_STATE, "mesh point count mismatch");
    min_unrefined = R.first();
}

namespace {

// test_panel (AMRStructure_amr.cpp:971-1081): flags a panel below max_height
// whose nine values meet a criterion: spread of f (eps0), spread relative to
// the centre value (eps1), max/min ratio (eps2), largest x difference quotient
// (eps3), p difference quotient (eps4: the reference reads six entries of
// which it sets two, the rest uninitialised; the two it sets are used).
bool test_panel(HostMesh& m, int pi, const std::vector<double>& f, const double* eps, int neps, int max_height) {
    HostPanel& P = m.panels[pi];
    double pf[9];
    for (int i = 0; i < 9; ++i) pf[i] = f[P.pts[i]];
    bool crit = false;
    if (neps > 0) {
        double mx = pf[0], mn = pf[0];
        for (int i = 1; i < 9; ++i) {
            if (mx < pf[i]) mx = pf[i];
            if (mn > pf[i]) mn = pf[i];
        }
        crit = crit || (mx - mn > eps[0]);
        if (neps > 1) crit = crit || (mx - mn) / pf[4] > eps[1];
        if (neps > 2) crit = crit || mx / mn > eps[2];
    }
    if (neps > 3) {
        const double dx = m.xs[P.pts[3]] - m.xs[P.pts[0]];
        double md = std::fabs((pf[3] - pf[0]) / dx);
        for (int i = 1; i < 6; ++i) {
            const double v = std::fabs((pf[3 + i] - pf[i]) / dx);
            if (md < v) md = v;
        }
        crit = crit || (md > eps[3]);
    }
    if (neps > 4) {
        const double dp = m.ps[P.pts[1]] - m.ps[P.pts[0]];
        double a[2] = {0.0, 0.0};
        for (int jj = 0; jj < 3; ++jj)
            for (int ii = 0; ii < 2; ++ii) a[ii] = std::fabs((pf[3 * jj + ii + 1] - pf[3 * jj + ii]) / dp);
        crit = crit || ((a[0] < a[1] ? a[1] : a[0]) > eps[4]);
    }
    if (P.level < max_height && crit) {
        P.needs = 1;
        return true;
    }
    return false;
}

}  // namespace

void HostMesh::restart_leaves() {
    leaves.clear();
    collect_leaves(*this, 0, leaves);
}

void HostMesh::adapt(std::vector<double>& f, const double* eps, int neps, int max_height,
                     const std::function<void(const double*, const double*, int, double*)>& eval) {
    Refiner R(*this);
    R.next_generation(min_unrefined);
    bool need = false;
    for (int i = min_unrefined; i < (int)panels.size(); ++i) need = test_panel(*this, i, f, eps, neps, max_height) || need;
    while (need) {
        need = false;
        R.need_further = false;
        const size_t n0 = xs.size();
        R.split_xp();
        need = R.need_further;
        f.resize(xs.size());
        if (xs.size() > n0) eval(xs.data() + n0, ps.data() + n0, (int)(xs.size() - n0), f.data() + n0);
        for (int i = min_unrefined; i < (int)panels.size(); ++i)
            if (!panels[i].xp) need = test_panel(*this, i, f, eps, neps, max_height) || need;
    }
    leaves.clear();
    collect_leaves(*this, 0, leaves);
}

// set_leaves_weights without the final *f (AMRStructure_amr.cpp:1084-1151):
// contributions are added leaf by leaf in DFS order, as in the reference.
std::vector<double> HostMesh::base_weights(double q, int quadrature) const {
    static const double trap[9] = {1.0, 2.0, 1.0, 2.0, 4.0, 2.0, 1.0, 2.0, 1.0};
    static const double simp[9] = {1.0, 4.0, 1.0, 4.0, 16.0, 4.0, 1.0, 4.0, 1.0};
    std::vector<double> w(xs.size(), 0.0);
    for (int l : leaves) {
        const HostPanel& P = panels[l];
        const double dx = xs[P.pts[3]] - xs[P.pts[0]];
        const double dp = ps[P.pts[1]] - ps[P.pts[0]];
        const bool simpson = (quadrature == 1);
        const double a = simpson ? q * dx * dp / 9.0 : q * dx * dp / 4.0;
        const double* st = simpson ? simp : trap;
        for (int i = 0; i < 9; ++i) w[P.pts[i]] += a * st[i];
    }
    return w;
}

void HostMesh::panel_records(int* out) const {
    for (size_t i = 0; i < panels.size(); ++i) {
        const HostPanel& P = panels[i];
        int* r = out + i * 18;
        for (int k = 0; k < 9; ++k) r[k] = P.pts[k];
        r[9] = P.level;
        r[10] = P.parent;
        r[11] = P.which;
        r[12] = P.child;
        r[13] = P.left;
        r[14] = P.top;
        r[15] = P.right;
        r[16] = P.bottom;
        r[17] = (P.lb ? 1 : 0) | (P.rb ? 2 : 0) | (P.xp ? 4 : 0) | (P.pr ? 8 : 0);
    }
}

// Initial distributions (distribution::operator() of the objects built by
// make_f0_return_ptr, AMRSimulation_load.cpp:139-225; initial_distributions.cpp).
// Evaluated on the host in the reference's operation order with the C library's
// exp/cos/sqrt, so the initial state is bit-identical to the reference's.  The
// reference evaluates the modified Bessel function K_1 and the incomplete
// elliptic integrals with Boost.Math; here they come from the C++17 standard
// library (std::cyl_bessel_k, std::ellint_1, std::ellint_2).
InitialDistribution::InitialDistribution(const fs_species_params& S, double xmin, double xmax)
    : ics(S.ics_type), pth(S.pth), pstr(S.pstr), amp(S.amp), mu(S.mu), wave_beta(S.wave_beta) {
    k = 2.0 * M_PI / (xmax - xmin) * S.normalized_wavenumber;
    switch (ics) {
        case 5: {  // F0_Friedman_beam(Delta = amp, Tstar = pth^2, xmax), :171-184, :241-262
            const double k_beta_0 = 2.0 * M_PI / 3.0, lambda_D = 2.81e-4, beta_b = 2.343e-3;
            const double gamma_b = 1.0 / std::sqrt(1 + beta_b * beta_b);
            fb_xcf = 1.0 / k_beta_0 / lambda_D / gamma_b;
            fb_nhat = 1.0 / (1.0 + amp);
            fb_pth = std::sqrt(pth * pth);
            const double dx = 0.01;
            const double nxd = std::ceil(1.1 * (xmax * fb_xcf) / dx);
            if (!(nxd >= 2) || nxd > 1e8) fail(FS_ERR_ARG, "Friedman beam: xmax gives no usable density table");
            const int nx = (int)nxd;
            fb_N.assign(nx, 0.0);
            fb_N[0] = 1.0;
            double Np = 0.0;  // dN/dx of the envelope equation, explicit Euler
            for (int i = 1; i < nx; ++i) {
                const double N0 = fb_N[i - 1];
                if (N0 <= 1e-150) continue;  // FRIEDMAN_BEAM_MIN_N: density stays 0
                fb_N[i] = N0 + dx * Np;
                Np += dx * (N0 * N0 - N0 * (1 + amp) + 1.0 / N0 * Np * Np);
            }
            fb_dx = 1 * dx - 0.0;  // xs[1] - xs[0] of the reference's table
            break;
        }
        case 6: case 7: {  // Maxwell_Jutner :306-313, Relativistic_Two_Stream :350-360
            if (!(mu > 0)) fail(FS_ERR_ARG, "relativistic initial condition needs mu > 0");
            k1mu = std::cyl_bessel_k(1.0, mu);
            if (!(k1mu > 0) || !std::isfinite(k1mu)) fail(FS_ERR_ARG, "K_1(mu) is not representable for this mu");
            gstr = std::sqrt(1 + pstr * pstr);
            break;
        }
        case 8: {  // Relativistic_Wave(amp, wave_beta, pth): check_gamma, make_cold_xs_ps, :366-433
            const double gm = amp;
            if (!(gm >= 1)) fail(FS_ERR_ARG, "relativistic wave: amp (the maximum gamma) must be >= 1");
            if (wave_beta < 1.0 && 1.0 / std::sqrt(1 - wave_beta * wave_beta) < gm)
                fail(FS_ERR_ARG, "relativistic wave: particles faster than the wave (max gamma above the wave's)");
            const double kap = std::sqrt((gm - 1.0) / (gm + 1.0));
            const double kap_p = std::sqrt(2 / (gm + 1.0));
            const int np = 100;
            const double da = 3 * M_PI / (np - 1);
            wv_x.resize(np);
            wv_p.resize(np);
            for (int i = 0; i < np; ++i) {
                const double a = -M_PI / 2 + i * da;
                const double x0 = wave_beta * (2 / kap_p * std::ellint_2(kap, a) - kap_p * std::ellint_1(kap, a));
                wv_x[i] = x0 + 2 * kap / kap_p * std::sin(a);
                const double g = gm - (gm - 1) * std::sin(a) * std::sin(a);
                wv_p[i] = std::sqrt(g * g - 1) * (std::cos(a) > 0 ? 1 : -1);
            }
            break;
        }
        default:  // any other value: F0_LD, like the reference's default branch
            break;
    }
}

double InitialDistribution::operator()(double x, double p) const {
    const double c = 1.0 / std::sqrt(2.0 * M_PI);
    switch (ics) {
        case 3: {  // F0_strong_two_stream: p^2 times the Landau seed with zero drift
            double seed = c / pth * std::exp(-(p - 0.0) * (p - 0.0) / 2 / pth / pth) * (1 + amp * std::cos(k * x));
            return seed * p * p;
        }
        case 4: {  // F0_colder_two_stream: two drifting Maxwellians
            double a = p - pstr, b = p + pstr;
            double ma = c / pth * std::exp(-(a - 0.0) * (a - 0.0) / 2 / pth / pth);
            double mb = c / pth * std::exp(-(b - 0.0) * (b - 0.0) / 2 / pth / pth);
            return .5 * (ma + mb) * (1 + amp * std::cos(k * x));
        }
        case 5: {  // Maxwellian in 1.25 p times the tabulated envelope at |x| / 1.25
            const double q = p * 1.25;
            const double m = c / fb_pth * std::exp(-(q - 0.0) * (q - 0.0) / 2 / fb_pth / fb_pth);
            const double u = std::fabs(x / 1.25) * fb_xcf / fb_dx;
            const double fl = std::floor(u);
            if (!(fl >= 0) || fl + 1 >= (double)fb_N.size())
                fail(FS_ERR_ARG, "Friedman beam: x beyond the tabulated density (1.1 xmax)");
            const int i = (int)fl;
            const double th = u - fl;
            return m * fb_nhat * ((1 - th) * fb_N[i] + th * fb_N[i + 1]);
        }
        case 6: {
            const double g = std::sqrt(1 + p * p);
            return std::exp(-g * mu) / 2.0 / k1mu * (1 + amp * std::cos(k * x));
        }
        case 7: {
            const double g = std::sqrt(1 + p * p);
            const double ppm = p * pstr * mu;
            const double ep = std::exp(ppm - gstr * g * mu) / 2.0 / k1mu;
            const double em = std::exp(-ppm - gstr * g * mu) / 2.0 / k1mu;
            return (ep + em) / 2.0 * (1 + amp * std::cos(k * x));
        }
        case 8: {  // thermal spread around the cold orbit, linear in x between table nodes
            if (!(x <= wv_x.back())) fail(FS_ERR_ARG, "relativistic wave: x beyond the tabulated orbit");
            size_t i = 0;
            while (x > wv_x[i + 1]) ++i;
            const double th = x - wv_x[i];  // not normalised by the node spacing, as in the reference
            const double p0 = (1 - th) * wv_p[i] + th * wv_p[i + 1];
            return 1.0 / std::sqrt(2 * M_PI) / pth * std::exp(-(p - p0) * (p - p0) / 2 / pth / pth);
        }
        default:  // 1, 2, 9, 10 (and unknown values): F0_LD, F0_ion_acoustic_electron/_ion share this form
            return c / pth * std::exp(-(p - pstr) * (p - pstr) / 2 / pth / pth) * (1 + amp * std::cos(k * x));
    }
}

}  // namespace fsb
