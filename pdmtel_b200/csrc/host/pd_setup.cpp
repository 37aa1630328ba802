// One-time host setup of the drop-in: Gauss rules, the cube-distance test,
// MLS contributors and coefficients.  Compiled with -ffp-contract=off; the
// operation order of every expression is the reference's, so the results are
// bit-identical to the reference's own setup (the golden-vector tests check
// this).  pow(x, 2.0), which g++ folds into x*x in the reference build, is
// written as x*x.
#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <thread>

#include "pdDataManager.h"

namespace pdh {

double Material::BulkSoundSpeed() const { return std::sqrt(BulkModulus() / density); }

bool Space::Contains(double x1, double x2, double x3, double tol) const {
    if (geo == 1)
        return x1 >= lo[0] - tol && x1 <= hi[0] + tol && x2 >= lo[1] - tol && x2 <= hi[1] + tol &&
               x3 >= lo[2] - tol && x3 <= hi[2] + tol;
    double dist = std::sqrt((x1 - c1) * (x1 - c1) + (x2 - c2) * (x2 - c2));
    return dist <= rad + tol && x3 >= lo[2] - tol && x3 <= hi[2] + tol;
}

// pdDataManager::SetGaussianPointsValue, pdDataManager3.cpp:1706-1799
void gauss_rule(int n, std::vector<double>& a, std::vector<double>& w) {
    a.clear();
    w.clear();
    switch (n) {
    case 2:
        a = {1.0 / std::sqrt(3.0), -1.0 / std::sqrt(3.0)};
        w = {1.0, 1.0};
        break;
    case 3:
        a = {0.0, std::sqrt(3.0 / 5.0), -std::sqrt(3.0 / 5.0)};
        w = {8.0 / 9.0, 5.0 / 9.0, 5.0 / 9.0};
        break;
    case 4: {
        const double s = std::sqrt(6.0 / 5.0);
        const double lo = std::sqrt((3.0 - 2.0 * s) / 7.0), hi = std::sqrt((3.0 + 2.0 * s) / 7.0);
        a = {lo, -lo, hi, -hi};
        const double wl = (18.0 + std::sqrt(30.0)) / 36.0, wh = (18.0 - std::sqrt(30.0)) / 36.0;
        w = {wl, wl, wh, wh};
        break;
    }
    case 5: {
        const double s = std::sqrt(10.0 / 7.0);
        const double lo = std::sqrt(5.0 - 2.0 * s) / 3.0, hi = std::sqrt(5.0 + 2.0 * s) / 3.0;
        a = {0.0, lo, -lo, hi, -hi};
        const double wl = (322.0 + 13.0 * std::sqrt(70.0)) / 900.0, wh = (322.0 - 13.0 * std::sqrt(70.0)) / 900.0;
        w = {128.0 / 225.0, wl, wl, wh, wh};
        break;
    }
    case 6: {
        // Gauss-Legendre n=6, each magnitude followed by its negative
        const double A[3] = {0.2386191860831969086305017, 0.6612093864662645136613996, 0.9324695142031520278123016};
        const double W[3] = {0.4679139345726910473898703, 0.3607615730481386075698335, 0.1713244923791703450402961};
        for (int k = 0; k < 3; ++k) {
            a.push_back(A[k]);
            a.push_back(-A[k]);
            w.push_back(W[k]);
            w.push_back(W[k]);
        }
        break;
    }
    case 8: {
        // Gauss-Legendre n=8: positive nodes, then the negatives
        const double A[4] = {0.1834346424956498049394761, 0.5255324099163289858177390, 0.7966664774136267395915539,
                             0.9602898564975362316835609};
        const double W[4] = {0.3626837833783619829651504, 0.3137066458778872873379622, 0.2223810344533744705443560,
                             0.1012285362903762591525314};
        for (int k = 0; k < 4; ++k) { a.push_back(A[k]); w.push_back(W[k]); }
        for (int k = 0; k < 4; ++k) { a.push_back(-A[k]); w.push_back(W[k]); }
        break;
    }
    default:
        a = {0.0};
        w = {2.0};
    }
}

namespace {

double shortest(double v, double lo, double hi, double tol) {
    if (v < lo - tol) return std::fabs(v - lo);
    if (v > hi + tol) return std::fabs(v - hi);
    return 0.0;
}

double longest(double v, double lo, double hi, double tol) {
    if (v < lo - tol) return std::fabs(v - hi);
    if (v > hi + tol) return std::fabs(v - lo);
    return (v > 0.5 * (hi + lo)) ? std::fabs(v - lo) : std::fabs(v - hi);
}

// distance from point pi to face `nrm` (1..3) at xf of the cube around pj;
// pdDataManager3.cpp:1573-1661
void face_distance(int nrm, double xf, const double* pi, const double* pj, double dx, double* dmn, double* dmx) {
    const double tol = 1e-4 * dx;
    const int n[3] = {nrm == 1, nrm == 2, nrm == 3};
    if (std::fabs((pi[0] - pj[0]) * n[0] + (pi[1] - pj[1]) * n[1] + (pi[2] - pj[2]) * n[2]) < tol) {
        *dmn = DBL_MAX;
        *dmx = DBL_MIN;
        return;
    }
    double lo[3], hi[3];
    for (int a = 0; a < 3; ++a) {
        lo[a] = pj[a] - 0.5 * dx;
        hi[a] = pj[a] + 0.5 * dx;
    }
    const double x_i = pi[0] * n[0] + pi[1] * n[1] + pi[2] * n[2];
    const double x_j = pj[0] * n[0] + pj[1] * n[1] + pj[2] * n[2];
    const double fac = (xf - x_i) / (x_j - x_i);
    double q[3];
    for (int a = 0; a < 3; ++a) q[a] = pi[a] + fac * (pj[a] - pi[a]);
    bool inside = true;
    for (int a = 0; a < 3; ++a) inside = inside && q[a] > lo[a] - tol && q[a] < hi[a] + tol;
    if (!inside) {
        *dmn = DBL_MAX;
        *dmx = DBL_MIN;
        return;
    }
    double foot[3], s[3], l[3];
    for (int a = 0; a < 3; ++a) foot[a] = (1 - n[a]) * pi[a] + n[a] * xf;
    for (int a = 0; a < 3; ++a) s[a] = (1 - n[a]) * shortest(foot[a], lo[a], hi[a], tol);
    for (int a = 0; a < 3; ++a) l[a] = (1 - n[a]) * longest(foot[a], lo[a], hi[a], tol);
    const double ffs = std::sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
    const double ffl = std::sqrt(l[0] * l[0] + l[1] * l[1] + l[2] * l[2]);
    const double itf = std::sqrt((foot[0] - pi[0]) * (foot[0] - pi[0]) + (foot[1] - pi[1]) * (foot[1] - pi[1]) +
                                 (foot[2] - pi[2]) * (foot[2] - pi[2]));
    *dmn = std::sqrt(ffs * ffs + itf * itf);
    *dmx = std::sqrt(ffl * ffl + itf * itf);
}

}  // namespace

// pdDataManager::CalcDistanceToCube, pdDataManager3.cpp:637-685
void cube_distance(const double* pi, const double* pj, double dx, double* dmin, double* dmax) {
    double mn = DBL_MAX, mx = DBL_MIN, a, b;
    for (int ax = 0; ax < 3; ++ax) {
        for (int side = 0; side < 2; ++side) {
            const double xf = side == 0 ? pj[ax] - 0.5 * dx : pj[ax] + 0.5 * dx;
            face_distance(ax + 1, xf, pi, pj, dx, &a, &b);
            mn = std::min(mn, a);
            mx = std::max(mx, b);
        }
    }
    *dmin = mn;
    *dmax = mx;
}

// pdDataManager::CalcBetaFactor, pdDataManager3.cpp:1801-1829
double beta_factor(double dist, double delta, double dx, bool cci_original) {
    const double inner = delta - 0.5 * dx;
    double outer = delta + 0.5 * dx;
    if (cci_original) outer = delta;
    if (dist <= inner) return 1.0;
    if (dist > inner && dist <= outer) return (delta + 0.5 * dx - dist) / dx;
    return 0.0;
}

// Contributors of each node: itself, then its family members within rw, or
// within 1.5 rw when fewer than 10 (the basis size) qualify;
// pdDataManager2.cpp:118-171.
int mls_contributors(int64_t n, const double* x, const int64_t* row_ptr, const int32_t* col, double rw,
                     std::vector<int64_t>& cb_ptr, std::vector<int32_t>& cb_idx) {
    cb_ptr.assign(n + 1, 0);
    cb_idx.clear();
    std::vector<int32_t> tmp;
    for (int64_t i = 0; i < n; ++i) {
        const double* pi = x + 3 * i;
        for (double radius : {rw, rw * 1.5}) {
            tmp.clear();
            tmp.push_back((int32_t)i);
            for (int64_t p = row_ptr[i]; p < row_ptr[i + 1]; ++p) {
                const double* pj = x + 3 * (int64_t)col[p];
                const double d1 = pj[0] - pi[0], d2 = pj[1] - pi[1], d3 = pj[2] - pi[2];
                if (std::sqrt(d1 * d1 + d2 * d2 + d3 * d3) <= radius) tmp.push_back(col[p]);
            }
            if (tmp.size() >= 10) break;
        }
        cb_idx.insert(cb_idx.end(), tmp.begin(), tmp.end());
        cb_ptr[i + 1] = (int64_t)cb_idx.size();
    }
    return PD_OK;
}

namespace {

// Quadratic basis [1 x y z xy xz yz x^2 y^2 z^2] in global coordinates,
// pdDataManager2.cpp:1547-1563
inline void basis(const double* q, double* p) {
    p[0] = 1.0;
    p[1] = q[0];
    p[2] = q[1];
    p[3] = q[2];
    p[4] = q[0] * q[1];
    p[5] = q[0] * q[2];
    p[6] = q[1] * q[2];
    p[7] = q[0] * q[0];
    p[8] = q[1] * q[1];
    p[9] = q[2] * q[2];
}

// quartic spline of |q - node| / rw, pdDataManager2.cpp:1565-1578
inline double spline_weight(const double* node, const double* q, double rw) {
    const double e1 = q[0] - node[0], e2 = q[1] - node[1], e3 = q[2] - node[2];
    const double r = std::sqrt(e1 * e1 + e2 * e2 + e3 * e3);
    const double d = r / rw;
    if (d > 1.0) return 0.0;
    return (1 - 6.0 * d * d + 8.0 * std::pow(d, 3.0) - 3.0 * std::pow(d, 4.0));
}

// Gauss-Jordan elimination with full pivoting on the 10x10 moment matrix in
// the operation order of pdMatrix::Gauss (pdMatrix.cpp:251-391).  The
// solution replaces rhs; the inverse bookkeeping (column unscrambling) is not
// needed for it and is skipped.
bool solve10(double A[10][10], double rhs[10]) {
    int piv[10] = {0};
    for (int step = 0; step < 10; ++step) {
        double big = 0.0;
        int prow = 0, pcol = 0;
        for (int r = 0; r < 10; ++r) {
            if (piv[r] == 1) continue;
            for (int cc = 0; cc < 10; ++cc) {
                if (piv[cc] == 0) {
                    if (std::fabs(A[r][cc]) >= big) {
                        big = std::fabs(A[r][cc]);
                        prow = r;
                        pcol = cc;
                    }
                } else if (piv[cc] > 1) {
                    return false;
                }
            }
        }
        ++piv[pcol];
        if (prow != pcol) {
            for (int cc = 0; cc < 10; ++cc) std::swap(A[prow][cc], A[pcol][cc]);
            std::swap(rhs[prow], rhs[pcol]);
        }
        if (A[pcol][pcol] == 0.0) return false;
        const double inv = 1.0 / A[pcol][pcol];
        A[pcol][pcol] = 1.0;
        for (int cc = 0; cc < 10; ++cc) A[pcol][cc] = A[pcol][cc] * inv;
        rhs[pcol] = rhs[pcol] * inv;
        for (int r = 0; r < 10; ++r) {
            if (r == pcol) continue;
            const double m = A[r][pcol];
            A[r][pcol] = 0.0;
            for (int cc = 0; cc < 10; ++cc) A[r][cc] = A[r][cc] - A[pcol][cc] * m;
            rhs[r] = rhs[r] + -m * rhs[pcol];
        }
    }
    return true;
}

}  // namespace

// MLS coefficients of node contributors cb [nc] at the global point q
// (pdDataManager2.cpp:173-256, pdIntgManager2.cpp:1879-1939): moment matrix
// sum_k w_k p_k p_k^T, solved against p(q), coefficient k = (w_k p_k) . sol.
// pw: scratch of 11 nc doubles.  False on a singular moment matrix.
bool mls_point(const double* x, const int32_t* cb, int64_t nc, const double q[3], double rw, double* pw,
               double* out) {
    double A[10][10] = {};
    for (int64_t k = 0; k < nc; ++k) {
        const double* node = x + 3 * (int64_t)cb[k];
        double* e = pw + 11 * k;
        basis(node, e);
        e[10] = spline_weight(node, q, rw);
        for (int r = 0; r < 10; ++r)
            for (int cc = 0; cc < 10; ++cc) A[r][cc] = A[r][cc] + e[10] * e[r] * e[cc];
    }
    double s[10];
    basis(q, s);
    if (!solve10(A, s)) return false;
    for (int64_t k = 0; k < nc; ++k) {
        const double* e = pw + 11 * k;
        double sum = 0.0;
        for (int r = 0; r < 10; ++r) sum += (e[r] * e[10]) * s[r];
        out[k] = sum;
    }
    return true;
}

// MLS shape coefficients of every Gauss point, pdDataManager2.cpp:173-256.
// Output per node: npt blocks of ncb values (the point's coefficient vector).
int mls_coefficients(int64_t n, const double* x, const double* abscis, int n1, double dx,
                     const std::vector<int64_t>& cb_ptr, const std::vector<int32_t>& cb_idx, double rw,
                     std::vector<double>& coeff, int nthreads, int64_t* bad_node) {
    const int npt = n1 * n1 * n1;
    coeff.assign((size_t)cb_ptr[n] * npt, 0.0);
    std::atomic<int64_t> next(0), bad(-1);
    auto worker = [&]() {
        std::vector<double> pw;  // per contributor: basis[10], weight
        for (;;) {
            const int64_t i0 = next.fetch_add(64);
            if (i0 >= n || bad.load() >= 0) return;
            const int64_t i1 = std::min<int64_t>(n, i0 + 64);
            for (int64_t i = i0; i < i1; ++i) {
                const int64_t b = cb_ptr[i], nc = cb_ptr[i + 1] - b;
                pw.resize((size_t)nc * 11);
                for (int g = 0; g < npt; ++g) {
                    const int gi = g / (n1 * n1), gj = (g / n1) % n1, gk = g % n1;
                    const double q[3] = {0.5 * dx * abscis[gi] + x[3 * i], 0.5 * dx * abscis[gj] + x[3 * i + 1],
                                         0.5 * dx * abscis[gk] + x[3 * i + 2]};
                    double* out = coeff.data() + b * npt + (int64_t)g * nc;
                    if (!mls_point(x, cb_idx.data() + b, nc, q, rw, pw.data(), out)) {
                        int64_t exp = -1;
                        bad.compare_exchange_strong(exp, i);
                        return;
                    }
                }
            }
        }
    };
    if (nthreads < 1) nthreads = 1;
    std::vector<std::thread> pool;
    for (int t = 1; t < nthreads; ++t) pool.emplace_back(worker);
    worker();
    for (auto& th : pool) th.join();
    if (bad.load() >= 0) {
        if (bad_node) *bad_node = bad.load();
        return PD_ERR_SINGULAR;
    }
    return PD_OK;
}

}  // namespace pdh
