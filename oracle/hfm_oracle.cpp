// CPU oracle of the GPU eikonal path: a restatement, in plain C++, of the
// reference's discrete scheme and of the drivers around it.
//
// TEST INFRASTRUCTURE.  Only tests/, __graft_entry__.smoke() and bench.py's
// CPU-baseline leg load this library, as a checker or as the timed CPU
// baseline; the product path never calls it.
//
// What is restated (reference files, paths inside the AGD project):
//   Selling decomposition, 2D    agd/Eikonal/HFM_CUDA/cuda/Geometry2.h:21-48
//   Selling decomposition, 3D    agd/Eikonal/HFM_CUDA/cuda/Geometry3.h:22-58
//   scalar product <x,m y>       cuda/Geometry_.h (scal_vmv)
//   sorting networks (n=2,3,6)   cuda/NetworkSort.h:17-60,363-373
//   neighbour values             cuda/HFM.h:28-138 (HFMNeighbors)
//   eikonal update + flow        cuda/HFM.h:142-208 (HFMUpdate)
//   tile visit                   cuda/Update.h:20-227, FiniteDifferences.h:17-106, HFMIter.h:10-86
//   FIM tile scheduling          cuda/Propagation.h:103-167; _solvers.py:94-120
//   geodesic ODE                 cuda/Kernel_GeodesicODE.h:164-412; _GetGeodesics.py:9-147
//   distance-to-seed map         cuda/Kernel_InfConvolution.h:66-92; _GetGeodesics.py:51-75
//   reverse AD linear system     _PostProcess.py:155-219 (solved here by ordered sweeps)
//   forward AD linear system     _PostProcess.py:181-191 (ordered sweeps)
//   source factorisation         cuda/EuclideanFactor.h:8-26, FiniteDifferences.h:30-75
//   second order scheme          cuda/HFM.h:91-138 (HFMNeighbors), 175-206 (weights)
//   wall visibility              cuda/Walls.h:12-50, FiniteDifferences.h:51-59
//
// Arrays passed to this library are in plain row-major grid layout (not the
// bilevel tile layout of the GPU kernels).  The tile structure is used only to
// reproduce the reference's visit schedule.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr int kIntMax = 2147483647;

template <class T> inline T inf() { return std::numeric_limits<T>::infinity(); }

// ---------------------------------------------------------------- Selling ---
// <x, m y> with m packed lower-triangular [m00, m10, m11, m20, m21, m22]; the
// products of integer offsets are formed in integer arithmetic and accumulated
// in T in the reference's order.
template <class T, int D>
T scal_vmv(const int *x, const T *m, const int *y) {
    T r = 0;
    int k = 0;
    for (int i = 0; i < D; ++i)
        for (int j = 0; j <= i; ++j, ++k)
            r += T(i == j ? x[i] * y[i] : x[i] * y[j] + x[j] * y[i]) * m[k];
    return r;
}

template <class T>
void selling2(const T *m, T w[3], int e[3][2]) {
    int sb[3][2] = {{1, 0}, {0, 1}, {-1, -1}};
    for (int iter = 0, red = 0; iter < 100 && red < 3; ++iter, ++red) {
        const int i = iter % 3, j = (iter + 1) % 3, k = (iter + 2) % 3;
        if (scal_vmv<T, 2>(sb[i], m, sb[j]) > 0) {
            for (int c = 0; c < 2; ++c) sb[k][c] = sb[i][c] - sb[j][c];
            for (int c = 0; c < 2; ++c) sb[i][c] = -sb[i][c];
            red = 0;
        }
    }
    for (int r = 0; r < 3; ++r) {
        const int i = r, j = (r + 1) % 3, k = (r + 2) % 3;
        w[r] = std::fmax(T(0), -scal_vmv<T, 2>(sb[i], m, sb[j]));
        e[r][0] = -sb[k][1];
        e[r][1] = sb[k][0];
    }
}

const int kPerm3[6][4] = {{0, 1, 2, 3}, {0, 2, 1, 3}, {0, 3, 1, 2}, {1, 2, 0, 3}, {1, 3, 0, 2}, {2, 3, 0, 1}};

template <class T>
void selling3(const T *m, T w[6], int e[6][3]) {
    int sb[4][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {-1, -1, -1}};
    for (int iter = 0, red = 0; iter < 100 && red < 6; ++iter, ++red) {
        const int *p = kPerm3[iter % 6];
        const int i = p[0], j = p[1];
        if (scal_vmv<T, 3>(sb[i], m, sb[j]) > 0) {
            const int k = p[2], l = p[3];
            for (int c = 0; c < 3; ++c) {
                sb[k][c] += sb[i][c];
                sb[l][c] += sb[i][c];
                sb[i][c] = -sb[i][c];
            }
            red = 0;
        }
    }
    for (int r = 0; r < 6; ++r) {
        const int *p = kPerm3[r];
        w[r] = std::fmax(T(0), -scal_vmv<T, 3>(sb[p[0]], m, sb[p[1]]));
        const int *a = sb[p[2]], *b = sb[p[3]];
        for (int c = 0; c < 3; ++c) {
            const int c1 = (c + 1) % 3, c2 = (c + 2) % 3;
            e[r][c] = a[c1] * b[c2] - a[c2] * b[c1];
        }
    }
}

// ------------------------------------------------------ sorting networks ---
template <class T>
inline void oswap(const T *v, int *o, int i, int j) {
    const int a = o[i], b = o[j];
    const bool lt = v[a] < v[b];
    o[i] = lt ? a : b;
    o[j] = lt ? b : a;
}
template <class T>
void sort_order(const T *v, int *o, int n) {
    for (int i = 0; i < n; ++i) o[i] = i;
    if (n == 2) {
        oswap(v, o, 0, 1);
    } else if (n == 3) {
        oswap(v, o, 1, 2); oswap(v, o, 0, 2); oswap(v, o, 0, 1);
    } else if (n == 6) {
        oswap(v, o, 1, 2); oswap(v, o, 4, 5);
        oswap(v, o, 0, 2); oswap(v, o, 3, 5);
        oswap(v, o, 0, 1); oswap(v, o, 3, 4); oswap(v, o, 2, 5);
        oswap(v, o, 0, 3); oswap(v, o, 1, 4);
        oswap(v, o, 2, 4); oswap(v, o, 1, 3);
        oswap(v, o, 2, 3);
    }
}

// -------------------------------------------------------------- problem ---
template <class T>
struct Problem {
    int D = 2, model = 0;  // model 0: isotropic, 1: Riemann, 2: diagonal, 3: Rander (Riemann + drift)
    int shape[3] = {1, 1, 1}, shape_i[3] = {1, 1, 1}, shape_o[3] = {1, 1, 1};
    int size_i = 1, size_o = 1;
    long size = 1;
    int nact = 2;
    T iso_w[3] = {0, 0, 0};
    // dual metric planes (Riemann), squared dual costs (diagonal), the inverse of
    // the quadratic part then the drift (Rander); grid layout
    const float *geom = nullptr;
    const float *rhs = nullptr;
    const unsigned char *seed = nullptr;
    // Source factorisation: within fact_r2 (squared, index units) of fact_origin,
    // neighbour values are shifted so that the scheme is exact for |x|_m, m the
    // metric at the seed (packed lower-triangular; isotropic: D diagonal entries).
    T fact_r2 = 0, fact_origin[3] = {0, 0, 0}, fact_m[6] = {0, 0, 0, 0, 0, 0};
    // Second order scheme (order: 2): threshold on |u - 2v + v2| / max(u - v); 0: off.
    T order2 = 0;
    // Walls: L1 distance to the nearest wall point (grid layout), 255 beyond the
    // bound; null: no walls.  A neighbour x + v with [x, x + v] blocked by a wall
    // has value +inf (and so has x + 2v at second order).
    const unsigned char *wall_dist = nullptr;

    int wdist(const int *y) const { return inside(y) ? int(wall_dist[flat(y)]) : 255; }
    // Whether the segment [x, x + v] meets no wall (Walls.h:18-50): clear far from
    // the walls or for |v|_1 below the wall distance at x; else walk the lattice
    // points round(k v / |v|_inf), k = 1..|v|_inf, rounding halves away from 0.
    bool visible(const int *x, const int *v) const {
        if (!wall_dist) return true;
        const int d0 = wdist(x);
        if (d0 == 255) return true;
        int l1 = 0, linf = 0;
        for (int c = 0; c < D; ++c) { l1 += std::abs(v[c]); linf = std::max(linf, std::abs(v[c])); }
        if (l1 < d0) return true;
        for (int k = 1; k <= linf; ++k) {
            int y[3], rest = 0;
            for (int c = 0; c < D; ++c) {
                const int num = v[c] * k;  // round(num / linf), halves away from zero
                const int w = num >= 0 ? (num + linf / 2) / linf : -((-num + linf / 2) / linf);
                rest += std::abs(v[c] - w);
                y[c] = x[c] + w;
            }
            const int d = wdist(y);
            if (rest < d) return true;
            if (d == 0) return false;
        }
        return true;
    }

    bool diagonal() const { return model == 0 || model == 2; }  // unit offsets
    T scal_fact(const T *x, const T *y) const {
        if (diagonal()) {
            T r = 0;
            for (int i = 0; i < D; ++i) r += fact_m[i] * x[i] * y[i];
            return r;
        }
        T r = 0;
        int k = 0;
        for (int i = 0; i < D; ++i)
            for (int j = 0; j <= i; ++j, ++k) r += (i == j ? x[i] * y[i] : x[i] * y[j] + x[j] * y[i]) * fact_m[k];
        return r;
    }
    // Shifts of the neighbour values at x - e_k (f[2k]) and x + e_k (f[2k+1]) of
    // grid point x (flat index n): the factorisation's, then the drift's
    // +<w, e_k> and -<w, e_k> (FiniteDifferences.h:41-45); f2 (or null): the
    // factorisation's shifts of x -/+ 2 e_k for the second order scheme (the
    // drift does not shift them).
    void shifts(const int *x, long n, int (*e)[3], T *f, T *f2 = nullptr) const {
        for (int k = 0; k < 2 * nact; ++k) f[k] = 0;
        if (f2)
            for (int k = 0; k < 2 * nact; ++k) f2[k] = 0;
        factor_shifts(x, e, f, f2);
        if (model == 3) {
            const int sd = D * (D + 1) / 2;
            for (int k = 0; k < nact; ++k) {
                T s = 0;
                for (int c = 0; c < D; ++c) s += T(geom[(sd + c) * size + n]) * T(e[k][c]);
                f[2 * k] += s;
                f[2 * k + 1] -= s;
            }
        }
    }
    void factor_shifts(const int *x, int (*e)[3], T *f, T *f2 = nullptr) const {
        if (!(fact_r2 > 0)) return;
        T xr[3] = {0, 0, 0}, r2 = 0;
        for (int c = 0; c < D; ++c) {
            xr[c] = T(x[c]) - fact_origin[c];
            r2 += xr[c] * xr[c];
        }
        if (!(r2 < fact_r2)) return;
        const T xx = scal_fact(xr, xr);
        for (int k = 0; k < nact; ++k) {
            T ek[3] = {0, 0, 0};
            for (int c = 0; c < D; ++c) ek[c] = T(e[k][c]);
            const T xe = scal_fact(xr, ek), ee = scal_fact(ek, ek);
            const T nx = std::sqrt(xx), nm = std::sqrt(xx - 2 * xe + ee), np = std::sqrt(xx + 2 * xe + ee);
            const T g = xe / nx;                       // <e, m x> / |x|_m
            const T d0 = (2 * xe - ee) / (nx + nm), d1 = (-2 * xe - ee) / (nx + np);  // |x| - |x-/+e|
            f[2 * k] = -g + d0;     // |x| - |x-e| - <e,mx>/|x|
            f[2 * k + 1] = g + d1;  // |x| - |x+e| + <e,mx>/|x|
            if (f2) {  // x -/+ 2e: the first order shift plus |x| - 2|x-/+e| + |x-/+2e| (EuclideanFactor.h:20-28)
                const T nm2 = std::sqrt(xx - 4 * xe + 4 * ee), np2 = std::sqrt(xx + 4 * xe + 4 * ee);
                f2[2 * k] = 2 * f[2 * k] - (d0 + (-2 * xe + 3 * ee) / (nm + nm2));
                f2[2 * k + 1] = 2 * f[2 * k + 1] - (d1 + (2 * xe + 3 * ee) / (np + np2));
            }
        }
    }

    void init(int D_, int model_, const int *shape_, const int *shape_i_) {
        D = D_;
        model = model_;
        size_i = 1;
        size_o = 1;
        size = 1;
        for (int k = 0; k < D; ++k) {
            shape[k] = shape_[k];
            shape_i[k] = shape_i_[k];
            shape_o[k] = (shape[k] + shape_i[k] - 1) / shape_i[k];
            size_i *= shape_i[k];
            size_o *= shape_o[k];
            size *= shape[k];
        }
        nact = diagonal() ? D : D * (D + 1) / 2;
    }
    long flat(const int *x) const {
        long n = 0;
        for (int k = 0; k < D; ++k) n = n * shape[k] + x[k];
        return n;
    }
    bool inside(const int *x) const {
        for (int k = 0; k < D; ++k)
            if (x[k] < 0 || x[k] >= shape[k]) return false;
        return true;
    }
    // Stencil at grid point n: weights w[nact], offsets e[nact][D].
    void stencil(long n, T *w, int (*e)[3]) const {
        if (diagonal()) {  // unit offsets; weights h^-2 (isotropic) or per point (diagonal, Isotropic_.h:32-36)
            for (int k = 0; k < D; ++k) {
                w[k] = model == 0 ? iso_w[k] : T(geom[k * size + n]);
                for (int c = 0; c < D; ++c) e[k][c] = (c == k);
            }
            return;
        }
        const int sd = D * (D + 1) / 2;
        T m[6];
        for (int c = 0; c < sd; ++c) m[c] = T(geom[c * size + n]);
        if (D == 2) {
            int e2[3][2];
            selling2<T>(m, w, e2);
            for (int r = 0; r < 3; ++r) { e[r][0] = e2[r][0]; e[r][1] = e2[r][1]; }
        } else {
            int e3[6][3];
            selling3<T>(m, w, e3);
            for (int r = 0; r < 6; ++r) for (int c = 0; c < 3; ++c) e[r][c] = e3[r][c];
        }
    }
};

// The eikonal update of one point from its neighbour values v[nact] (each the
// smaller of the two symmetric neighbours).  Returns the candidate value and,
// optionally, the upwind flow weights.
template <class T>
T hfm_update(T rhs, const T *w, const T *v, int nact, T *flow_w) {
    int o[6];
    sort_order(v, o, nact);
    const T vmin = v[o[0]];
    if (vmin == inf<T>()) {
        if (flow_w) for (int k = 0; k < nact; ++k) flow_w[k] = 0;
        return vmin;
    }
    T a = w[o[0]], b = 0, c = -rhs * rhs;
    for (int q = 1; q < nact; ++q) {
        const int k = o[q];
        const T t = v[k] - vmin;
        if ((a * t - 2 * b) * t + c > 0) break;
        a += w[k];
        b += w[k] * t;
        c += w[k] * t * t;
    }
    const T delta = b * b - a * c;
    const T sd = std::sqrt(std::fmax(T(0), delta));
    const T value = a == T(0) ? inf<T>() : (b + sd) / a;
    const T val = vmin + value;
    if (flow_w) {
        if (val == inf<T>()) {
            for (int k = 0; k < nact; ++k) flow_w[k] = 0;
        } else {
            for (int k = 0; k < nact; ++k) flow_w[k] = w[k] * std::fmax(T(0), val - v[k]);
        }
    }
    return val;
}

// Second order corrections (HFM.h:91-138): u0 the point's value, v[k] the
// smaller of the two neighbours along e_k (on side[k]), v2[k] the neighbour two
// steps away on that side.  Where |u0 - 2 v + v2| < thr * max_k (u0 - v_k) and
// u0 > v, v becomes v + (v - v2) / 3 and o2[k] = 1 (weight x 9/4, flow x 3/2).
template <class T>
void order2_correct(T u0, T *v, const T *v2, int nact, T thr, char *o2) {
    T bound = 0;
    for (int k = 0; k < nact; ++k) bound = std::max(bound, u0 - v[k]);
    for (int k = 0; k < nact; ++k) {
        const T d2 = std::fabs(u0 - 2 * v[k] + v2[k]);
        o2[k] = d2 < thr * bound && u0 > v[k];
        // v + (v - v2) / 3 with the quotient and the sum in double, rounded once
        // (the reference divides by the double literal 3., HFM.h:129)
        if (o2[k]) v[k] = T(double(v[k]) + double(v[k] - v2[k]) / 3.0);
    }
}

// ------------------------------------------------------------ tile visit ---
template <class T>
struct Solver {
    Problem<T> P;
    std::vector<T> u;  // grid layout values
    T atol = 0, rtol = 0;
    int niter_i = 8, front = 4;

    // Grid indices of the points of tile n_o (-1 for padding) and their in-tile coordinates.
    void tile_points(int n_o, long *pts, int *xi, int *xt) const {
        int xo[3];
        int r = n_o;
        for (int k = P.D - 1; k >= 0; --k) { xo[k] = r % P.shape_o[k]; r /= P.shape_o[k]; }
        for (int n_i = 0; n_i < P.size_i; ++n_i) {
            int q = n_i;
            for (int k = P.D - 1; k >= 0; --k) {
                xi[n_i * 3 + k] = q % P.shape_i[k];
                q /= P.shape_i[k];
                xt[n_i * 3 + k] = xo[k] * P.shape_i[k] + xi[n_i * 3 + k];
            }
            pts[n_i] = P.inside(xt + n_i * 3) ? P.flat(xt + n_i * 3) : -1;
        }
    }

    // One visit of tile n_o (Update.h:20-227): returns true if some point of the
    // tile moved by more than atol + rtol |u|.
    bool visit(int n_o) {
        const int S = P.size_i, NA = P.nact, D = P.D;
        std::vector<long> pts(S);
        std::vector<int> xi(3 * S), xt(3 * S);
        tile_points(n_o, pts.data(), xi.data(), xt.data());
        std::vector<T> ul(S), uold(S), rhs(S), w(S * 6), vo(S * 12), sh(S * 12, T(0)), vo2(S * 12), sh2(S * 12, T(0));
        std::vector<int> vi(S * 12), vi2(S * 12);
        std::vector<char> seed(S);
        for (int n = 0; n < S; ++n) {
            const long p = pts[n];
            if (p < 0) {  // padding: a seed whose right-hand side is +inf
                ul[n] = uold[n] = inf<T>();
                seed[n] = 1;
                continue;
            }
            uold[n] = u[p];
            seed[n] = P.seed[p] != 0;
            rhs[n] = T(P.rhs[p]);
            ul[n] = seed[n] ? rhs[n] : uold[n];
            int e[6][3];
            P.stencil(p, &w[n * 6], e);
            if (!seed[n]) P.shifts(xt.data() + n * 3, p, e, &sh[n * 12], P.order2 > 0 ? &sh2[n * 12] : nullptr);
            for (int k = 0; k < NA; ++k)
                for (int s = 0; s < 2; ++s) {
                    const int ks = 2 * k + s, eps = 2 * s - 1;
                    int yi[3], yt[3], off[3] = {0, 0, 0};
                    bool intile = true;
                    for (int c = 0; c < D; ++c) {
                        off[c] = eps * e[k][c];
                        yi[c] = xi[n * 3 + c] + off[c];
                        yt[c] = xt[n * 3 + c] + off[c];
                        if (yi[c] < 0 || yi[c] >= P.shape_i[c]) intile = false;
                    }
                    if (!seed[n] && !P.visible(xt.data() + n * 3, off)) {  // hidden by a wall
                        vi[n * 12 + ks] = vi2[n * 12 + ks] = -1;
                        vo[n * 12 + ks] = vo2[n * 12 + ks] = inf<T>();
                        continue;
                    }
                    if (intile) {
                        int li = 0;
                        for (int c = 0; c < D; ++c) li = li * P.shape_i[c] + yi[c];
                        vi[n * 12 + ks] = li;
                    } else {
                        vi[n * 12 + ks] = -1;
                        vo[n * 12 + ks] = P.inside(yt) ? u[P.flat(yt)] : inf<T>();
                    }
                    if (P.order2 > 0) {  // the neighbour two steps away
                        bool in2 = true;
                        for (int c = 0; c < D; ++c) {
                            yi[c] += eps * e[k][c];
                            yt[c] += eps * e[k][c];
                            if (yi[c] < 0 || yi[c] >= P.shape_i[c]) in2 = false;
                        }
                        if (in2) {
                            int li = 0;
                            for (int c = 0; c < D; ++c) li = li * P.shape_i[c] + yi[c];
                            vi2[n * 12 + ks] = li;
                        } else {
                            vi2[n * 12 + ks] = -1;
                            vo2[n * 12 + ks] = P.inside(yt) ? u[P.flat(yt)] : inf<T>();
                        }
                    }
                }
        }
        for (int it = 0; it < niter_i; ++it) {
            bool moved = false;
            for (int n = 0; n < S; ++n) {
                if (seed[n]) continue;
                T v[6], v2[6], wk[6];
                int side[6];
                for (int k = 0; k < NA; ++k) {
                    T best = 0;
                    side[k] = 0;
                    for (int s = 0; s < 2; ++s) {
                        const int ks = 2 * k + s;
                        const T val = (vi[n * 12 + ks] >= 0 ? ul[vi[n * 12 + ks]] : vo[n * 12 + ks]) + sh[n * 12 + ks];
                        if (s == 0) best = val;
                        else if (best > val) { best = val; side[k] = 1; }
                    }
                    v[k] = best;
                    wk[k] = w[n * 6 + k];
                }
                if (P.order2 > 0) {
                    for (int k = 0; k < NA; ++k) {
                        const int ks = 2 * k + side[k];
                        v2[k] = (vi2[n * 12 + ks] >= 0 ? ul[vi2[n * 12 + ks]] : vo2[n * 12 + ks]) + sh2[n * 12 + ks];
                    }
                    char o2[6];
                    order2_correct<T>(ul[n], v, v2, NA, P.order2, o2);
                    for (int k = 0; k < NA; ++k)
                        if (o2[k]) wk[k] *= T(9) / T(4);
                }
                const T cand = hfm_update<T>(rhs[n], wk, v, NA, nullptr);
                if (ul[n] > cand) { ul[n] = cand; moved = true; }
            }
            if (!moved) break;  // a pass without change is a fixed point of the visit
        }
        bool changed = false;
        for (int n = 0; n < S; ++n) {
            if (pts[n] < 0) continue;
            u[pts[n]] = ul[n];
            const T diff = std::fabs(uold[n] - ul[n]);
            const T tol = atol + rtol * std::fabs(ul[n]);
            if (!(std::isnan(diff) || diff <= tol)) changed = true;
        }
        return changed;
    }

    void tile_neighbors(int n_o, int *nb, int &cnt) const {
        int xo[3], r = n_o;
        for (int k = P.D - 1; k >= 0; --k) { xo[k] = r % P.shape_o[k]; r /= P.shape_o[k]; }
        cnt = 0;
        for (int q = 0; q < 2 * P.D; ++q) {
            int y[3] = {xo[0], xo[1], xo[2]};
            y[q / 2] += 2 * (q % 2) - 1;
            bool ok = true;
            for (int k = 0; k < P.D; ++k) ok = ok && y[k] >= 0 && y[k] < P.shape_o[k];
            if (!ok) { nb[q] = -1; continue; }
            int m = 0;
            for (int k = 0; k < P.D; ++k) m = m * P.shape_o[k] + y[k];
            nb[q] = m;
            ++cnt;
        }
    }

    // Fast iterative method over tiles (_solvers.py:94-120, Propagation.h:103-167).
    int fim(const unsigned char *trigger_tiles, int nitermax, int nthreads, long long *visits) {
        const int SO = P.size_o;
        std::vector<unsigned char> upd(trigger_tiles, trigger_tiles + SO), sA(SO, 0), sB(SO, 0);
        unsigned char *sPrev = sA.data(), *sNext = sB.data();
        std::vector<int> list;
        long long nvis = 0;
        int niter = 0;
        for (; niter < nitermax; ++niter) {
            list.clear();
            for (int n = 0; n < SO; ++n) if (upd[n]) list.push_back(n);
            if (list.empty()) break;
            std::swap(sPrev, sNext);
            std::fill(upd.begin(), upd.end(), 0);
            std::fill(sNext, sNext + SO, 0);
            const int L = (int)list.size();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads) if (nthreads > 1)
            for (int b = 0; b < L; ++b) {
                const int n_o = list[b];
                const bool changed = visit(n_o);
                int nb[6], cnt;
                tile_neighbors(n_o, nb, cnt);
                const unsigned char scoreFront = (unsigned char)front, sp = sPrev[n_o];
                bool propagate;
                int scoreNext;
                if (!changed) {
                    if (sp == 0 || sp == scoreFront) { scoreNext = 0; propagate = false; }
                    else { scoreNext = scoreFront; propagate = true; }
                } else {
                    scoreNext = 1;
                    upd[n_o] = 1;
                    if (scoreFront > 2)
                        for (int q = 0; q < 2 * P.D; ++q)
                            scoreNext = std::max(scoreNext, (nb[q] >= 0 ? (int)sPrev[nb[q]] : 0) - 1);
                    propagate = scoreNext > 1;
                }
                sNext[n_o] = (unsigned char)scoreNext;
                if (propagate)
                    for (int q = 0; q < 2 * P.D; ++q) if (nb[q] >= 0) upd[nb[q]] = 1;
            }
            nvis += L;
        }
        if (visits) *visits = nvis;
        return niter;
    }

    // Upwind flow at every point from the converged values (the flow variant of
    // Update.h:171-209 with one local iteration).  Values are refreshed in place
    // by that iteration, like the reference's flow pass.
    void flow(T *fvec, T *fwsum, T *fw, int *fidx) {
        const int NA = P.nact, D = P.D;
        const long N = P.size;
        std::vector<T> unew(u);
        for (long p = 0; p < N; ++p) {
            int x[3];
            long q = p;
            for (int k = D - 1; k >= 0; --k) { x[k] = int(q % P.shape[k]); q /= P.shape[k]; }
            T wts[6] = {0, 0, 0, 0, 0, 0};
            int side[6] = {0, 0, 0, 0, 0, 0};
            int e[6][3];
            const bool sd = P.seed[p] != 0;
            if (!sd) {
                P.stencil(p, wts, e);
                T v[6], sh[12], sh2[12];
                P.shifts(x, p, e, sh, sh2);
                bool hid[12];
                for (int k = 0; k < NA; ++k) {
                    for (int s = 0; s < 2; ++s) {
                        int y[3], off[3] = {0, 0, 0};
                        for (int c = 0; c < D; ++c) off[c] = (2 * s - 1) * e[k][c];
                        for (int c = 0; c < D; ++c) y[c] = x[c] + off[c];
                        hid[2 * k + s] = !P.visible(x, off);
                        const T val = (!hid[2 * k + s] && P.inside(y) ? u[P.flat(y)] : inf<T>()) + sh[2 * k + s];
                        if (s == 0) { v[k] = val; side[k] = 0; }
                        else if (v[k] > val) { v[k] = val; side[k] = 1; }
                    }
                }
                T f[6], wk[6];
                char o2[6] = {0, 0, 0, 0, 0, 0};
                for (int k = 0; k < NA; ++k) wk[k] = wts[k];
                if (P.order2 > 0) {
                    T v2[6];
                    for (int k = 0; k < NA; ++k) {
                        int y[3];
                        for (int c = 0; c < D; ++c) y[c] = x[c] + 2 * (2 * side[k] - 1) * e[k][c];
                        v2[k] = (!hid[2 * k + side[k]] && P.inside(y) ? u[P.flat(y)] : inf<T>()) + sh2[2 * k + side[k]];
                    }
                    order2_correct<T>(u[p], v, v2, NA, P.order2, o2);
                    for (int k = 0; k < NA; ++k)
                        if (o2[k]) wk[k] *= T(9) / T(4);
                }
                const T cand = hfm_update<T>(T(P.rhs[p]), wk, v, NA, f);
                if (u[p] > cand) unew[p] = cand;
                for (int k = 0; k < NA; ++k)  // flow weights from the plain weights, x 3/2 at second order
                    wts[k] = cand == inf<T>() ? T(0) : wts[k] * std::fmax(T(0), cand - v[k]) * (o2[k] ? T(1.5) : T(1));
            } else {
                P.stencil(p, wts, e);
                for (int k = 0; k < NA; ++k) wts[k] = 0;
                unew[p] = T(P.rhs[p]);
            }
            T vec[3] = {0, 0, 0}, sum = 0;
            for (int k = 0; k < NA; ++k) {
                sum += wts[k];
                const int eps = 2 * side[k] - 1;
                int y[3];
                for (int c = 0; c < D; ++c) {
                    const int off = eps * e[k][c];
                    vec[c] += wts[k] * T(off);
                    y[c] = x[c] + off;
                }
                if (fw) fw[k * N + p] = wts[k];
                if (fidx) fidx[k * N + p] = wts[k] != T(0) ? int(P.flat(y)) : kIntMax;
            }
            for (int c = 0; c < D; ++c) fvec[c * N + p] = vec[c];
            fwsum[p] = sum;
        }
        u.swap(unew);
    }
};

// ------------------------------------------------------------ geodesics ---
enum { kContinue = 0, kAtSeed, kInWall, kStationnary, kPastSeed, kVanishingFlow };

template <class T>
struct Geodesic {
    int D;
    const int *shape;
    long N;
    const T *u, *fvec, *fwsum;
    const unsigned char *eucl;
    T step, causality;
    int eucl_delay, nymin_delay;

    bool inside(const int *y) const {
        for (int k = 0; k < D; ++k) if (y[k] < 0 || y[k] >= shape[k]) return false;
        return true;
    }
    long flat(const int *y) const {
        long n = 0;
        for (int k = 0; k < D; ++k) n = n * shape[k] + y[k];
        return n;
    }

    struct Cache {
        int xq[3];
        long nymin;
        T thr;
        T flow[8][3], dist[8], wsum[8];
    };

    // Interpolated, causality filtered, normalised flow (Kernel_GeodesicODE.h:164-260).
    int normalized_flow(const T *x, T *flow, Cache &c) const {
        const int nc = 1 << D;
        bool newcell = false;
        for (int k = 0; k < D; ++k) {
            const int q = int(std::floor(x[k]));
            if (q != c.xq[k]) newcell = true;
            c.xq[k] = q;
        }
        T dx[3], wts[8];
        for (int k = 0; k < D; ++k) dx[k] = x[k] - T(c.xq[k]);
        for (int i = 0; i < nc; ++i) {
            wts[i] = 1;
            for (int k = 0; k < D; ++k) wts[i] *= ((i >> k) & 1) ? dx[k] : T(1) - dx[k];
        }
        if (newcell) {
            for (int i = 0; i < nc; ++i) {
                int y[3];
                for (int k = 0; k < D; ++k) y[k] = c.xq[k] + ((i >> k) & 1);
                if (!inside(y)) { c.dist[i] = inf<T>(); continue; }
                const long n = flat(y);
                c.dist[i] = u[n];
                c.wsum[i] = fwsum[n];
                for (int k = 0; k < D; ++k) c.flow[i][k] = fvec[k * N + n];
            }
            T dmin = inf<T>();
            int imin = -1;
            const T wthr = T(0.5) / T(nc);
            for (int i = 0; i < nc; ++i) {
                if (wts[i] < wthr) continue;
                if (c.dist[i] < dmin) { imin = i; dmin = c.dist[i]; }
            }
            if (dmin == inf<T>()) return kInWall;
            int y[3];
            for (int k = 0; k < D; ++k) y[k] = c.xq[k] + ((imin >> k) & 1);
            c.nymin = flat(y);
            if (c.wsum[imin] == T(0)) return kAtSeed;
            c.thr = dmin + causality / c.wsum[imin];
        }
        for (int k = 0; k < D; ++k) flow[k] = 0;
        for (int i = 0; i < nc; ++i) {
            if (c.dist[i] >= c.thr) continue;
            for (int k = 0; k < D; ++k) flow[k] += wts[i] * c.flow[i][k];
        }
        T n2 = 0;
        for (int k = 0; k < D; ++k) n2 += flow[k] * flow[k];
        const T nrm = std::sqrt(n2);
        if (!(nrm > 0)) return kVanishingFlow;
        const T l = T(1.0 / double(nrm));
        for (int k = 0; k < D; ++k) flow[k] *= l;
        return kContinue;
    }

    // One backtracking chunk of at most max_len points from x_s[0] (Kernel_GeodesicODE.h:265-412).
    int chunk(T *x_s, int max_len, int pastseed_delay, int *len_out) const {
        const int hlen = 1 + std::max(eucl_delay, nymin_delay);
        std::vector<unsigned char> eucl_p(hlen, 255);
        std::vector<long> nymin_p(hlen, (long)kIntMax);
        Cache c;
        for (int k = 0; k < 3; ++k) c.xq[k] = kIntMax;
        c.nymin = kIntMax;
        c.thr = 0;
        T x[3];
        for (int k = 0; k < D; ++k) x[k] = x_s[k];
        int len, stop = kContinue;
        for (len = 1; len < max_len; ++len) {
            const int l = len % hlen;
            T xp[3], xm[3], flow[3];
            for (int k = 0; k < D; ++k) xp[k] = x[k];
            stop = normalized_flow(x, flow, c);
            if (stop != kContinue) break;
            nymin_p[l] = c.nymin;
            eucl_p[l] = eucl[c.nymin];
            if (c.nymin == nymin_p[(l - nymin_delay + hlen) % hlen]) { stop = kStationnary; break; }
            // The reference's subscript here is a boolean expression (value 0 or 1).
            const int cmp = (((l - eucl_delay + hlen) % hlen) != 0) && (len >= pastseed_delay);
            if (eucl_p[l] > eucl_p[cmp]) { stop = kPastSeed; break; }
            for (int k = 0; k < D; ++k) xm[k] = (T(0.5) * step) * flow[k] + xp[k];
            stop = normalized_flow(xm, flow, c);
            if (stop != kContinue) break;
            for (int k = 0; k < D; ++k) x[k] = step * flow[k] + xp[k];
            for (int k = 0; k < D; ++k) x_s[len * D + k] = x[k];
        }
        *len_out = len;
        return stop;
    }
};

// Min-plus distance-to-seed map in units of 1/5 pixel, saturated at 255, six
// passes of a 3^d kernel, then cut beyond 30 (_GetGeodesics.py:51-75).
void eucl_map(int D, const int *shape, const unsigned char *seedmask, unsigned char *out) {
    long N = 1;
    for (int k = 0; k < D; ++k) N *= shape[k];
    std::vector<unsigned char> a(N), b(N);
    for (long p = 0; p < N; ++p) a[p] = seedmask[p] ? 0 : 255;
    const int nk = D == 2 ? 9 : 27;
    for (int it = 0; it < 6; ++it) {
        for (long p = 0; p < N; ++p) {
            int x[3];
            long q = p;
            for (int k = D - 1; k >= 0; --k) { x[k] = int(q % shape[k]); q /= shape[k]; }
            int best = 255;
            for (int ic = 0; ic < nk; ++ic) {
                int y[3], r = ic, n2 = 0;
                bool ok = true;
                for (int k = D - 1; k >= 0; --k) {
                    const int o = r % 3 - 1;
                    r /= 3;
                    y[k] = x[k] + o;
                    n2 += o * o;
                    ok = ok && y[k] >= 0 && y[k] < shape[k];
                }
                if (!ok) continue;
                long m = 0;
                for (int k = 0; k < D; ++k) m = m * shape[k] + y[k];
                const int kv = int(std::lround(5.0 * std::sqrt(double(n2))));
                const int av = a[m];
                const int s = (av >= 255 - kv) ? 255 : av + kv;
                best = std::min(best, s);
            }
            b[p] = (unsigned char)best;
        }
        a.swap(b);
    }
    for (long p = 0; p < N; ++p) out[p] = a[p] > 30 ? 255 : a[p];
}

template <class T>
void fill_problem(Problem<T> &P, int ndim, int model, const int *shape, const int *shape_i,
                  const double *iso_w, const float *geom, const float *rhs, const unsigned char *seed) {
    P.init(ndim, model, shape, shape_i);
    for (int k = 0; k < ndim; ++k) P.iso_w[k] = iso_w ? T(iso_w[k]) : T(0);
    P.geom = geom;
    P.rhs = rhs;
    P.seed = seed;
}

// Source factorisation of the next solves (agdo_set_factor).
double g_fact_r2 = 0, g_fact_origin[3] = {0, 0, 0}, g_fact_m[6] = {0, 0, 0, 0, 0, 0};
double g_order2 = 0;
const unsigned char *g_wall_dist = nullptr;  // walls of the next solves (agdo_set_walls)

template <class T>
int eikonal_impl(int ndim, int model, const int *shape, const int *shape_i, int niter_i, int front,
                 const double *iso_w, const float *geom, const float *rhs, const unsigned char *seed,
                 double *values, double atol, double rtol, int nitermax, int nthreads,
                 long long *visits, double *fvec, double *fwsum, double *fw, int *fidx) {
    Solver<T> S;
    fill_problem(S.P, ndim, model, shape, shape_i, iso_w, geom, rhs, seed);
    S.P.fact_r2 = T(g_fact_r2);
    for (int c = 0; c < 3; ++c) S.P.fact_origin[c] = T(g_fact_origin[c]);
    for (int c = 0; c < 6; ++c) S.P.fact_m[c] = T(g_fact_m[c]);
    S.P.order2 = T(g_order2);
    S.P.wall_dist = g_wall_dist;
    S.u.assign(values, values + S.P.size);
    S.atol = T(atol);
    S.rtol = T(rtol);
    S.niter_i = niter_i;
    S.front = front;
    std::vector<unsigned char> trig(S.P.size_o, 0);
    for (long p = 0; p < S.P.size; ++p) {  // the tiles of the seeds, walls excluded (_SetArgs.py:119-126)
        if (!seed[p] || (g_wall_dist && g_wall_dist[p] == 0)) continue;
        int x[3], n_o = 0;
        long q = p;
        for (int k = ndim - 1; k >= 0; --k) { x[k] = int(q % shape[k]); q /= shape[k]; }
        for (int k = 0; k < ndim; ++k) n_o = n_o * S.P.shape_o[k] + x[k] / shape_i[k];
        trig[n_o] = 1;
    }
    const int niter = S.fim(trig.data(), nitermax, nthreads, visits);
    if (fvec) {
        const long N = S.P.size;
        std::vector<T> v(ndim * N), s(N), w(S.P.nact * N);
        S.flow(v.data(), s.data(), w.data(), fidx);
        for (long i = 0; i < ndim * N; ++i) fvec[i] = v[i];
        for (long i = 0; i < N; ++i) fwsum[i] = s[i];
        if (fw) for (long i = 0; i < S.P.nact * N; ++i) fw[i] = w[i];
    }
    for (long p = 0; p < S.P.size; ++p) values[p] = S.u[p];
    return niter;
}

}  // namespace

extern "C" {

// Selling decomposition of n packed symmetric matrices (symdim floats each).
void agdo_selling_f32(int ndim, const float *m, int n, float *w, int *e) {
    for (int p = 0; p < n; ++p) {
        if (ndim == 2) {
            float ww[3]; int ee[3][2];
            selling2<float>(m + 3 * p, ww, ee);
            for (int r = 0; r < 3; ++r) { w[3 * p + r] = ww[r]; e[(3 * p + r) * 2] = ee[r][0]; e[(3 * p + r) * 2 + 1] = ee[r][1]; }
        } else {
            float ww[6]; int ee[6][3];
            selling3<float>(m + 6 * p, ww, ee);
            for (int r = 0; r < 6; ++r) { w[6 * p + r] = ww[r]; for (int c = 0; c < 3; ++c) e[(6 * p + r) * 3 + c] = ee[r][c]; }
        }
    }
}

// Eikonal solve on the grid layout.  `values` holds the initial values (+inf for a
// cold start) and receives the solution; arithmetic in float (dbl=0) or double.
// With fvec non-null the upwind flow is exported too (vector: ndim planes,
// weightsum, weights and grid-flat indices: nact planes, INT_MAX when inactive).
int agdo_eikonal(int dbl, int ndim, int model, const int *shape, const int *shape_i, int niter_i,
                 int front, const double *iso_w, const float *geom, const float *rhs,
                 const unsigned char *seed, double *values, double atol, double rtol, int nitermax,
                 int nthreads, long long *visits, double *fvec, double *fwsum, double *fw,
                 int *fidx) {
    if (dbl)
        return eikonal_impl<double>(ndim, model, shape, shape_i, niter_i, front, iso_w, geom, rhs, seed,
                                    values, atol, rtol, nitermax, nthreads, visits, fvec, fwsum, fw, fidx);
    return eikonal_impl<float>(ndim, model, shape, shape_i, niter_i, front, iso_w, geom, rhs, seed, values,
                               atol, rtol, nitermax, nthreads, visits, fvec, fwsum, fw, fidx);
}

// Walls for the following agdo_eikonal calls: wall distances in grid layout
// (0 at the walls, 255 far from them), kept by pointer; NULL: no walls.  The
// walls must also be seeds of right-hand side +inf in those calls.
void agdo_set_walls(const unsigned char *wall_dist) { g_wall_dist = wall_dist; }

// Second order scheme for the following agdo_eikonal calls (threshold; 0: off).
void agdo_set_order2(double threshold) { g_order2 = threshold; }

// Source factorisation for the following agdo_eikonal calls (r2 = 0: off).
void agdo_set_factor(double r2, const double *origin, const double *metric) {
    g_fact_r2 = r2;
    for (int c = 0; c < 3; ++c) g_fact_origin[c] = origin ? origin[c] : 0.0;
    for (int c = 0; c < 6; ++c) g_fact_m[c] = metric ? metric[c] : 0.0;
}

void agdo_eucl_map(int ndim, const int *shape, const unsigned char *seedmask, unsigned char *out) {
    eucl_map(ndim, shape, seedmask, out);
}

// One geodesic chunk per tip (float arithmetic, like the reference kernel).
// x_s: (ntips, max_len, ndim) with x_s[:,0] the start points (continuous indices).
void agdo_geodesic_chunk(int ndim, const int *shape, int ntips, int max_len, int pastseed_delay,
                         float causality, float step, int eucl_delay, int nymin_delay, const float *u,
                         const float *fvec, const float *fwsum, const unsigned char *eucl, float *x_s,
                         int *len_s, signed char *stop_s) {
    Geodesic<float> G;
    G.D = ndim;
    G.shape = shape;
    G.N = 1;
    for (int k = 0; k < ndim; ++k) G.N *= shape[k];
    G.u = u; G.fvec = fvec; G.fwsum = fwsum; G.eucl = eucl;
    G.step = step; G.causality = causality;
    G.eucl_delay = eucl_delay; G.nymin_delay = nymin_delay;
    for (int t = 0; t < ntips; ++t) {
        int len;
        stop_s[t] = (signed char)G.chunk(x_s + (long)t * max_len * ndim, max_len, pastseed_delay, &len);
        len_s[t] = len;
    }
}

// Forward linearisation (agd/Eikonal/HFM_CUDA/_PostProcess.py:181-191):
// fwsum(x) du(x) - sum_k fw_k(x) du(y_k(x)) = rhs(x), diag 1 where fwsum = 0.
// The upwind neighbours y_k(x) have smaller values than x, so Gauss-Seidel
// sweeps in increasing order of the values settle in one pass (a second one
// confirms; ties are harmless).
int agdo_forward(int nact, long N, const double *values, const double *fw, const int *fidx,
                 const double *fwsum, const double *rhs, double *du) {
    std::vector<long> order(N);
    for (long i = 0; i < N; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](long a, long b) {
        const double va = std::isfinite(values[a]) ? values[a] : 1e300;
        const double vb = std::isfinite(values[b]) ? values[b] : 1e300;
        return va < vb;
    });
    for (long i = 0; i < N; ++i) du[i] = 0;
    int sweeps = 0;
    for (; sweeps < 1000; ++sweeps) {
        double maxchg = 0, maxval = 0;
        for (long q = 0; q < N; ++q) {
            const long x = order[q];
            double acc = rhs[x];
            for (int k = 0; k < nact; ++k) {
                const double w = fw[k * N + x];
                const int y = fidx[k * N + x];
                if (w != 0 && y != kIntMax && y >= 0 && y < N) acc += w * du[y];
            }
            const double d = fwsum[x] == 0 ? 1.0 : fwsum[x];
            const double nv = acc / d;
            maxchg = std::max(maxchg, std::fabs(nv - du[x]));
            maxval = std::max(maxval, std::fabs(nv));
            du[x] = nv;
        }
        if (maxchg <= 1e-15 * std::max(1.0, maxval)) break;
    }
    return sweeps;
}

// Reverse-mode sensitivity: solves diag(x) lam(x) - sum_{z->x} w lam(z) = s(x)
// (transpose of the linearised scheme, _PostProcess.py:155-219) where the entries
// z->x are the upwind weights fw[k][z] with fidx[k][z] == x.  diag = weightsum,
// or 1 where weightsum == 0.  Points are swept by decreasing value, repeated
// until nothing moves, in double precision.
int agdo_reverse(int nact, long N, const double *values, const double *fw, const int *fidx,
                 const double *fwsum, const double *sens, double *lam) {
    std::vector<long> cnt(N + 1, 0);
    for (int k = 0; k < nact; ++k)
        for (long z = 0; z < N; ++z)
            if (fw[k * N + z] != 0 && fidx[k * N + z] != kIntMax) cnt[fidx[k * N + z] + 1]++;
    for (long i = 0; i < N; ++i) cnt[i + 1] += cnt[i];
    std::vector<long> src(cnt[N]);
    std::vector<double> wt(cnt[N]);
    std::vector<long> fill(cnt.begin(), cnt.end() - 1);
    for (int k = 0; k < nact; ++k)
        for (long z = 0; z < N; ++z) {
            const double w = fw[k * N + z];
            const int x = fidx[k * N + z];
            if (w != 0 && x != kIntMax) { src[fill[x]] = z; wt[fill[x]] = w; fill[x]++; }
        }
    std::vector<long> order(N);
    for (long i = 0; i < N; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](long a, long b) {
        const double va = std::isfinite(values[a]) ? values[a] : -1e300;
        const double vb = std::isfinite(values[b]) ? values[b] : -1e300;
        return va > vb;
    });
    for (long i = 0; i < N; ++i) lam[i] = 0;
    int sweeps = 0;
    for (; sweeps < 1000; ++sweeps) {
        double maxchg = 0, maxval = 0;
        for (long q = 0; q < N; ++q) {
            const long x = order[q];
            double acc = sens[x];
            for (long j = cnt[x]; j < cnt[x + 1]; ++j) acc += wt[j] * lam[src[j]];
            const double d = fwsum[x] == 0 ? 1.0 : fwsum[x];
            const double nv = acc / d;
            maxchg = std::max(maxchg, std::fabs(nv - lam[x]));
            maxval = std::max(maxval, std::fabs(nv));
            lam[x] = nv;
        }
        if (maxchg <= 1e-15 * std::max(1.0, maxval)) break;
    }
    return sweeps;
}

}  // extern "C"
