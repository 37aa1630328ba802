/*
 * pd_oracle.c — CPU restatement of the pdMTEL hot path (test infrastructure;
 * see pd_oracle.h).  Compile with -O2 -ffp-contract=off: every expression
 * below keeps the reference's evaluation order, and pow(x, 2.0), which g++
 * folds into x*x in the reference build, is written as x*x.
 */
#include "pd_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define OR_PI acos(-1.0)   /* pdIntgManager.h:25 */
#define OR_MEGA DBL_MAX    /* pdIntgManager.h:26 */
#define OR_TINY DBL_MIN    /* pdIntgManager.h:27 */

static double dmin2(double a, double b) { return (b < a) ? b : a; }
static double dmax2(double a, double b) { return (a < b) ? b : a; }

/* ---------------------------------------------------------------- Gauss -- */

int or_gauss_1d(int n, double* a, double* w) {
    switch (n) {
    case 2:
        a[0] = 1.0 / sqrt(3.0); a[1] = -1.0 / sqrt(3.0);
        w[0] = 1.0; w[1] = 1.0;
        return 2;
    case 3:
        a[0] = 0.0; a[1] = sqrt(3.0 / 5.0); a[2] = -sqrt(3.0 / 5.0);
        w[0] = 8.0 / 9.0; w[1] = 5.0 / 9.0; w[2] = 5.0 / 9.0;
        return 3;
    case 4: {
        double s = sqrt(6.0 / 5.0);
        a[0] = sqrt((3.0 - 2.0 * s) / 7.0); a[1] = -sqrt((3.0 - 2.0 * s) / 7.0);
        a[2] = sqrt((3.0 + 2.0 * s) / 7.0); a[3] = -sqrt((3.0 + 2.0 * s) / 7.0);
        w[0] = (18.0 + sqrt(30.0)) / 36.0; w[1] = w[0];
        w[2] = (18.0 - sqrt(30.0)) / 36.0; w[3] = w[2];
        return 4;
    }
    case 5: {
        double s = sqrt(10.0 / 7.0);
        a[0] = 0.0;
        a[1] = sqrt(5.0 - 2.0 * s) / 3.0; a[2] = -sqrt(5.0 - 2.0 * s) / 3.0;
        a[3] = sqrt(5.0 + 2.0 * s) / 3.0; a[4] = -sqrt(5.0 + 2.0 * s) / 3.0;
        w[0] = 128.0 / 225.0;
        w[1] = (322.0 + 13.0 * sqrt(70.0)) / 900.0; w[2] = w[1];
        w[3] = (322.0 - 13.0 * sqrt(70.0)) / 900.0; w[4] = w[3];
        return 5;
    }
    case 6: {
        /* Gauss-Legendre n=6 nodes/weights, listed +,- per magnitude */
        static const double A[3] = {0.2386191860831969086305017, 0.6612093864662645136613996,
                                    0.9324695142031520278123016};
        static const double W[3] = {0.4679139345726910473898703, 0.3607615730481386075698335,
                                    0.1713244923791703450402961};
        for (int k = 0; k < 3; ++k) { a[2 * k] = A[k]; a[2 * k + 1] = -A[k]; w[2 * k] = W[k]; w[2 * k + 1] = W[k]; }
        return 6;
    }
    case 8: {
        /* Gauss-Legendre n=8: the four positive nodes, then their negatives */
        static const double A[4] = {0.1834346424956498049394761, 0.5255324099163289858177390,
                                    0.7966664774136267395915539, 0.9602898564975362316835609};
        static const double W[4] = {0.3626837833783619829651504, 0.3137066458778872873379622,
                                    0.2223810344533744705443560, 0.1012285362903762591525314};
        for (int k = 0; k < 4; ++k) { a[k] = A[k]; a[k + 4] = -A[k]; w[k] = W[k]; w[k + 4] = W[k]; }
        return 8;
    }
    default:
        a[0] = 0.0; w[0] = 2.0;
        return 1;
    }
}

void or_gauss_points(int64_t n, const double* x, double dx, int n1, double* xg, double* gw) {
    double a[8], w[8];
    int m = or_gauss_1d(n1, a, w);
    int npt = m * m * m;
    for (int i = 0; i < m; ++i)
        for (int j = 0; j < m; ++j)
            for (int k = 0; k < m; ++k) {
                int g = (i * m + j) * m + k;
                gw[3 * g] = w[i]; gw[3 * g + 1] = w[j]; gw[3 * g + 2] = w[k];
            }
    for (int64_t p = 0; p < n; ++p)
        for (int i = 0; i < m; ++i)
            for (int j = 0; j < m; ++j)
                for (int k = 0; k < m; ++k) {
                    int g = (i * m + j) * m + k;
                    double* q = xg + (p * npt + g) * 3;
                    q[0] = 0.5 * dx * a[i] + x[3 * p];
                    q[1] = 0.5 * dx * a[j] + x[3 * p + 1];
                    q[2] = 0.5 * dx * a[k] + x[3 * p + 2];
                }
}

/* ------------------------------------------------------- bond search --- */

static double shortest_between(double v, double lo, double hi, double tol) {
    if (v < lo - tol) return fabs(v - lo);
    else if (v > hi + tol) return fabs(v - hi);
    return 0.0;
}

static double longest_between(double v, double lo, double hi, double tol) {
    if (v < lo - tol) return fabs(v - hi);
    else if (v > hi + tol) return fabs(v - lo);
    if (v > 0.5 * (hi + lo)) return fabs(v - lo);
    return fabs(v - hi);
}

/* pdDataManager3.cpp:1573-1661 */
static void dist_to_face(int nrm, double xf, const double* pi, const double* pj, double dx,
                         double* dmin, double* dmax) {
    double tol = 1e-4 * dx;
    int n1 = nrm == 1, n2 = nrm == 2, n3 = nrm == 3;
    double xi1 = pi[0], xi2 = pi[1], xi3 = pi[2];
    double xj1 = pj[0], xj2 = pj[1], xj3 = pj[2];
    if (fabs((xi1 - xj1) * n1 + (xi2 - xj2) * n2 + (xi3 - xj3) * n3) < tol) {
        *dmin = OR_MEGA; *dmax = OR_TINY;
        return;
    }
    double x1lo = xj1 - 0.5 * dx, x1hi = xj1 + 0.5 * dx;
    double x2lo = xj2 - 0.5 * dx, x2hi = xj2 + 0.5 * dx;
    double x3lo = xj3 - 0.5 * dx, x3hi = xj3 + 0.5 * dx;
    double x_i = xi1 * n1 + xi2 * n2 + xi3 * n3;
    double x_j = xj1 * n1 + xj2 * n2 + xj3 * n3;
    double fac = (xf - x_i) / (x_j - x_i);
    double x1int = xi1 + fac * (xj1 - xi1);
    double x2int = xi2 + fac * (xj2 - xi2);
    double x3int = xi3 + fac * (xj3 - xi3);
    if (x1int > x1lo - tol && x1int < x1hi + tol && x2int > x2lo - tol && x2int < x2hi + tol &&
        x3int > x3lo - tol && x3int < x3hi + tol) {
        double f1 = (1 - n1) * xi1 + n1 * xf;
        double f2 = (1 - n2) * xi2 + n2 * xf;
        double f3 = (1 - n3) * xi3 + n3 * xf;
        double s1 = (1 - n1) * shortest_between(f1, x1lo, x1hi, tol);
        double s2 = (1 - n2) * shortest_between(f2, x2lo, x2hi, tol);
        double s3 = (1 - n3) * shortest_between(f3, x3lo, x3hi, tol);
        double l1 = (1 - n1) * longest_between(f1, x1lo, x1hi, tol);
        double l2 = (1 - n2) * longest_between(f2, x2lo, x2hi, tol);
        double l3 = (1 - n3) * longest_between(f3, x3lo, x3hi, tol);
        double ffs = sqrt(s1 * s1 + s2 * s2 + s3 * s3);
        double ffl = sqrt(l1 * l1 + l2 * l2 + l3 * l3);
        double itf = sqrt((f1 - xi1) * (f1 - xi1) + (f2 - xi2) * (f2 - xi2) + (f3 - xi3) * (f3 - xi3));
        *dmin = sqrt(ffs * ffs + itf * itf);
        *dmax = sqrt(ffl * ffl + itf * itf);
        return;
    }
    *dmin = OR_MEGA; *dmax = OR_TINY;
}

/* pdDataManager3.cpp:637-685; pi is the lower-id node of the pair */
static void dist_to_cube(const double* pi, const double* pj, double dx, double* mn, double* mx) {
    double a, b;
    *mn = OR_MEGA; *mx = OR_TINY;
    double lo[3] = {pj[0] - 0.5 * dx, pj[1] - 0.5 * dx, pj[2] - 0.5 * dx};
    double hi[3] = {pj[0] + 0.5 * dx, pj[1] + 0.5 * dx, pj[2] + 0.5 * dx};
    for (int ax = 0; ax < 3; ++ax) {
        dist_to_face(ax + 1, lo[ax], pi, pj, dx, &a, &b);
        *mn = dmin2(*mn, a); *mx = dmax2(*mx, b);
        dist_to_face(ax + 1, hi[ax], pi, pj, dx, &a, &b);
        *mn = dmin2(*mn, a); *mx = dmax2(*mx, b);
    }
}

static int cmp_i32(const void* a, const void* b) {
    int32_t x = *(const int32_t*)a, y = *(const int32_t*)b;
    return (x > y) - (x < y);
}

int64_t or_bond_search(int64_t n, const double* x, double dx, double delta, int64_t* row_ptr,
                       int32_t* col, int64_t cap, double* min_bond) {
    double tol = 1.0e-4 * dx;
    /* cell binning only narrows the candidate pairs; membership is decided
     * by the reference's exact cube-distance test */
    double lo[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, hi[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
    for (int64_t i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a) { lo[a] = dmin2(lo[a], x[3 * i + a]); hi[a] = dmax2(hi[a], x[3 * i + a]); }
    double h = delta + dx;
    int64_t nc[3];
    for (int a = 0; a < 3; ++a) nc[a] = (int64_t)floor((hi[a] - lo[a]) / h) + 1;
    int64_t ncell = nc[0] * nc[1] * nc[2];
    int64_t* cstart = (int64_t*)calloc((size_t)ncell + 1, sizeof(int64_t));
    int64_t* cell = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n ? n : 1));
    int64_t* order = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n ? n : 1));
    int32_t* buf = NULL;
    int64_t bufcap = 0;
    for (int64_t i = 0; i < n; ++i) {
        int64_t c[3];
        for (int a = 0; a < 3; ++a) c[a] = (int64_t)floor((x[3 * i + a] - lo[a]) / h);
        cell[i] = (c[2] * nc[1] + c[1]) * nc[0] + c[0];
        cstart[cell[i] + 1]++;
    }
    for (int64_t c = 0; c < ncell; ++c) cstart[c + 1] += cstart[c];
    {
        int64_t* fill = (int64_t*)malloc(sizeof(int64_t) * (size_t)(ncell + 1));
        memcpy(fill, cstart, sizeof(int64_t) * (size_t)(ncell + 1));
        for (int64_t i = 0; i < n; ++i) order[fill[cell[i]]++] = i;
        free(fill);
    }
    double mb = delta;
    int64_t total = 0;
    row_ptr[0] = 0;
    for (int64_t i = 0; i < n; ++i) {
        int64_t ci = cell[i];
        int64_t cx = ci % nc[0], cy = (ci / nc[0]) % nc[1], cz = ci / (nc[0] * nc[1]);
        int64_t cnt = 0;
        for (int64_t dz = -1; dz <= 1; ++dz)
            for (int64_t dy = -1; dy <= 1; ++dy)
                for (int64_t dxc = -1; dxc <= 1; ++dxc) {
                    int64_t qx = cx + dxc, qy = cy + dy, qz = cz + dz;
                    if (qx < 0 || qy < 0 || qz < 0 || qx >= nc[0] || qy >= nc[1] || qz >= nc[2]) continue;
                    int64_t q = (qz * nc[1] + qy) * nc[0] + qx;
                    for (int64_t s = cstart[q]; s < cstart[q + 1]; ++s) {
                        int64_t j = order[s];
                        if (j == i) continue;
                        int64_t a = i < j ? i : j, b = i < j ? j : i;
                        const double* pa = x + 3 * a;
                        const double* pb = x + 3 * b;
                        double dmn, dmx;
                        dist_to_cube(pa, pb, dx, &dmn, &dmx);
                        if (dmn < delta + tol) {
                            if (cnt >= bufcap) {
                                bufcap = bufcap ? 2 * bufcap : 1024;
                                buf = (int32_t*)realloc(buf, sizeof(int32_t) * (size_t)bufcap);
                            }
                            buf[cnt++] = (int32_t)j;
                            if (i < j) {
                                double d1 = pb[0] - pa[0], d2 = pb[1] - pa[1], d3 = pb[2] - pa[2];
                                double dist = sqrt(d1 * d1 + d2 * d2 + d3 * d3);
                                mb = dmin2(mb, dist);
                            }
                        }
                    }
                }
        if (col) {
            if (total + cnt > cap) { total = -1; break; }
            qsort(buf, (size_t)cnt, sizeof(int32_t), cmp_i32);
            memcpy(col + total, buf, sizeof(int32_t) * (size_t)cnt);
        }
        total += cnt;
        row_ptr[i + 1] = total;
    }
    if (min_bond) *min_bond = mb;
    free(cstart); free(cell); free(order); free(buf);
    return total;
}

/* ------------------------------------------------------------- slit ---- */

/* Project rule (the reference's pdSlit is data only): the rectangle's normal
 * axis is its thinnest extent; a bond is deleted iff its end points lie
 * strictly on opposite sides of that plane and the crossing point lies inside
 * the other two extents (inclusive). */
static int slit_crosses(const double* s, const double* a, const double* b) {
    int nrm = 0;
    double ext = s[1] - s[0];
    for (int k = 1; k < 3; ++k)
        if (s[2 * k + 1] - s[2 * k] < ext) { ext = s[2 * k + 1] - s[2 * k]; nrm = k; }
    double c = 0.5 * (s[2 * nrm] + s[2 * nrm + 1]);
    double da = a[nrm] - c, db = b[nrm] - c;
    if (!((da < 0.0 && db > 0.0) || (da > 0.0 && db < 0.0))) return 0;
    double t = (c - a[nrm]) / (b[nrm] - a[nrm]);
    for (int k = 0; k < 3; ++k) {
        if (k == nrm) continue;
        double p = a[k] + t * (b[k] - a[k]);
        if (p < s[2 * k] || p > s[2 * k + 1]) return 0;
    }
    return 1;
}

void or_slit_mark(int64_t n, const double* x, const int64_t* row_ptr, const int32_t* col, int nslit,
                  const double* slits, uint8_t* broken) {
    for (int64_t i = 0; i < n; ++i)
        for (int64_t p = row_ptr[i]; p < row_ptr[i + 1]; ++p) {
            int64_t j = col[p];
            /* the segment is always taken from the lower id to the higher id */
            const double* a = x + 3 * (i < j ? i : j);
            const double* b = x + 3 * (i < j ? j : i);
            uint8_t br = 0;
            for (int s = 0; s < nslit; ++s) br |= (uint8_t)slit_crosses(slits + 6 * s, a, b);
            broken[p] = br;
        }
}

/* -------------------------------------------------------------- MLS ---- */

int64_t or_mls_contributors(int64_t n, const double* x, const int64_t* row_ptr, const int32_t* col,
                            double rw, int64_t* cb_ptr, int32_t* cb_idx) {
    int64_t total = 0;
    cb_ptr[0] = 0;
    for (int64_t i = 0; i < n; ++i) {
        const double* pi = x + 3 * i;
        int64_t cnt = 1;
        for (int pass = 0; pass < 2; ++pass) {
            double r = pass == 0 ? rw : rw * 1.5;
            cnt = 1;
            if (cb_idx) cb_idx[total] = (int32_t)i;
            for (int64_t p = row_ptr[i]; p < row_ptr[i + 1]; ++p) {
                const double* pj = x + 3 * (int64_t)col[p];
                double d1 = pj[0] - pi[0], d2 = pj[1] - pi[1], d3 = pj[2] - pi[2];
                double dist = sqrt(d1 * d1 + d2 * d2 + d3 * d3);
                if (dist <= r) {
                    if (cb_idx) cb_idx[total + cnt] = col[p];
                    ++cnt;
                }
            }
            if (cnt >= 10) break; /* BASISDIM, pdDataManager.h:37 */
        }
        total += cnt;
        cb_ptr[i + 1] = total;
    }
    return total;
}

static void basis10(double x, double y, double z, double* p) {
    p[0] = 1.0; p[1] = x; p[2] = y; p[3] = z;
    p[4] = x * y; p[5] = x * z; p[6] = y * z;
    p[7] = x * x; p[8] = y * y; p[9] = z * z;
}

static double mls_weight(const double* node, double x, double y, double z, double rw) {
    double xi1 = x - node[0], xi2 = y - node[1], xi3 = z - node[2];
    double r = sqrt(xi1 * xi1 + xi2 * xi2 + xi3 * xi3);
    double d = r / rw;
    if (d > 1.0) return 0.0;
    return (1 - 6.0 * d * d + 8.0 * pow(d, 3.0) - 3.0 * pow(d, 4.0));
}

/* Gauss-Jordan with full pivoting in the operation order of
 * pdMatrix.cpp:251-391; only the solution is kept. */
static int gauss_jordan10(double a[10][10], double b[10]) {
    int ipiv[10] = {0}, irow = 0, icol = 0;
    for (int i = 0; i < 10; ++i) {
        double big = 0.0;
        for (int j = 0; j < 10; ++j) {
            if (ipiv[j] != 1) {
                for (int k = 0; k < 10; ++k) {
                    if (ipiv[k] == 0) {
                        if (fabs(a[j][k]) >= big) { big = fabs(a[j][k]); irow = j; icol = k; }
                    } else if (ipiv[k] > 1) {
                        return -1;
                    }
                }
            }
        }
        ++ipiv[icol];
        if (irow != icol) {
            for (int l = 0; l < 10; ++l) { double t = a[irow][l]; a[irow][l] = a[icol][l]; a[icol][l] = t; }
            double t = b[irow]; b[irow] = b[icol]; b[icol] = t;
        }
        if (a[icol][icol] == 0.0) return -2;
        double pivinv = 1.0 / a[icol][icol];
        a[icol][icol] = 1.0;
        for (int l = 0; l < 10; ++l) a[icol][l] = a[icol][l] * pivinv;
        b[icol] = b[icol] * pivinv;
        for (int ll = 0; ll < 10; ++ll) {
            if (ll != icol) {
                double dum = a[ll][icol];
                a[ll][icol] = 0.0;
                for (int l = 0; l < 10; ++l) a[ll][l] = a[ll][l] - a[icol][l] * dum;
                b[ll] = b[ll] + -dum * b[icol];
            }
        }
    }
    return 0;
}

int64_t or_mls_coeff(int64_t n, const double* x, const double* xg, int npt, const int64_t* cb_ptr,
                     const int32_t* cb_idx, double rw, double* coeff) {
    double* pw = NULL;
    int64_t pwcap = 0;
    for (int64_t i = 0; i < n; ++i) {
        int64_t nc = cb_ptr[i + 1] - cb_ptr[i];
        const int32_t* cb = cb_idx + cb_ptr[i];
        if (nc * 11 > pwcap) { pwcap = nc * 11; pw = (double*)realloc(pw, sizeof(double) * (size_t)pwcap); }
        for (int g = 0; g < npt; ++g) {
            const double* q = xg + (i * npt + g) * 3;
            double a[10][10];
            memset(a, 0, sizeof(a));
            for (int64_t k = 0; k < nc; ++k) {
                const double* pk = x + 3 * (int64_t)cb[k];
                double p[10];
                basis10(pk[0], pk[1], pk[2], p);
                double w = mls_weight(pk, q[0], q[1], q[2], rw);
                for (int r = 0; r < 10; ++r)
                    for (int c = 0; c < 10; ++c) a[r][c] = a[r][c] + w * p[r] * p[c];
                memcpy(pw + 11 * k, p, sizeof(p));
                pw[11 * k + 10] = w;
            }
            double s[10];
            basis10(q[0], q[1], q[2], s);
            if (gauss_jordan10(a, s) != 0) { free(pw); return -(i + 1); }
            double* out = coeff + cb_ptr[i] * npt + (int64_t)g * nc;
            for (int64_t k = 0; k < nc; ++k) {
                double sum = 0.0;
                for (int r = 0; r < 10; ++r) sum += (pw[11 * k + r] * pw[11 * k + 10]) * s[r];
                out[k] = sum;
            }
        }
    }
    free(pw);
    return 0;
}

/* ------------------------------------------------- bonds and forces ---- */

/* pdDataManager3.cpp:1801-1829 */
static double beta_factor(double dist, double delta, double dx, int cci, int cci_mdf) {
    double inner = delta - 0.5 * dx;
    double outer = delta + 0.5 * dx;
    if (cci && !cci_mdf) outer = delta;
    if (dist <= inner) return 1.0;
    else if (dist > inner && dist <= outer) return (delta + 0.5 * dx - dist) / dx;
    return 0.0;
}

/* pdDataManager2.cpp:1293-1351 */
static void bond_force(const or_model* m, const double* xi, const double* eta, double ecrit, double spring,
                       double be, double effw, double* f, double* elast) {
    double r = sqrt(xi[0] * xi[0] + xi[1] * xi[1] + xi[2] * xi[2]);
    double y1 = xi[0] + eta[0], y2 = xi[1] + eta[1], y3 = xi[2] + eta[2];
    double p = sqrt(y1 * y1 + y2 * y2 + y3 * y3);
    double dxe = effw * m->dx / 2.0;
    double beta = beta_factor(r, m->delta, dxe, m->cci, m->cci_mdf);
    double u = p - r;
    double s = u / r;
    if (u <= 0.0 || (u > 0.0 && s <= ecrit)) {
        if (m->cci) {
            double vol = m->dx * m->dx * m->dx;
            f[0] = be * vol * beta * spring * s * (xi[0] + eta[0]) / p;
            f[1] = be * vol * beta * spring * s * (xi[1] + eta[1]) / p;
            f[2] = be * vol * beta * spring * s * (xi[2] + eta[2]) / p;
        } else {
            f[0] = be * beta * spring * s * (xi[0] + eta[0]) / p;
            f[1] = be * beta * spring * s * (xi[1] + eta[1]) / p;
            f[2] = be * beta * spring * s * (xi[2] + eta[2]) / p;
        }
        *elast = be * 0.5 * (0.5 * beta * (spring / r) * u * u) * pow(0.5 * effw, 3);
    } else {
        f[0] = f[1] = f[2] = 0.0;
        *elast = 0.0;
    }
}

static double time_factor(const or_model* m, int b, double t) {
    if (m->bc_type[b] == OR_VELOC) return (t <= m->bc_end[b]) ? 1.0 : 0.0;
    if (m->bc_load[b] == 1.0) return (t <= m->bc_end[b]) ? t / m->bc_end[b] : 1.0;
    return 1.0;
}

static double pair_spring(const or_model* m, int64_t i, int64_t j) {
    double ci = m->mat_spring[m->mat[i]], cj = m->mat_spring[m->mat[j]];
    double c = (cj < ci) ? cj : ci; /* std::min(ci, cj) */
    if (m->spring_factor) c = c * (0.5 * (m->spring_factor[i] + m->spring_factor[j]));
    return c;
}

/* pdDataManager.cpp:2497-2602 */
static void update_node_bc(or_model* m, double t) {
    for (int64_t i = 0; i < m->n; ++i) {
        int b = m->bc[i];
        if (b < 0) continue;
        int ty = m->bc_type[b];
        const int32_t* dir = m->bc_dir + 3 * b;
        const double* v = m->bc_val + 9 * b;
        double fac = time_factor(m, b, t);
        const double* X = m->x + 3 * i;
        for (int a = 0; a < 3; ++a) {
            if (dir[a] != 1) continue;
            if (ty == OR_DISPL) {
                m->U[3 * i + a] = v[a] * fac;
                m->vbuf[3 * i + a] = 0.0;
            } else if (ty == OR_VELOC) {
                m->vbuf[3 * i + a] = v[a] * fac;
            } else if (ty == OR_DISPLGRAD) {
                m->U[3 * i + a] = (v[3 * a] * X[0] + v[3 * a + 1] * X[1] + v[3 * a + 2] * X[2]) * fac;
                m->vbuf[3 * i + a] = 0.0;
            }
        }
    }
}

void or_force_stage(or_model* m, double dts, double t, const double* us, double* k) {
    double vol8 = pow(m->dx, 3) / 8.0;
    for (int64_t i = 0; i < m->n; ++i) {
        int mi = m->mat[i];
        double rho = m->mat_density[mi];
        double body[3] = {m->mat_grav[3 * mi] * rho, m->mat_grav[3 * mi + 1] * rho, m->mat_grav[3 * mi + 2] * rho};
        const double* ui = (m->bc[i] >= 0) ? m->U + 3 * i : us + 3 * i;
        const double* xi = m->x + 3 * i;
        for (int64_t p = m->fam_ptr[i]; p < m->fam_ptr[i + 1]; ++p) {
            if (m->broken && m->broken[p]) continue;
            int64_t j = m->fam_col[p];
            int mj = m->mat[j];
            double ecrit = (m->mat_ecrit[mj] < m->mat_ecrit[mi]) ? m->mat_ecrit[mj] : m->mat_ecrit[mi];
            double spring = pair_spring(m, i, j);
            double be = 0.5 * (m->bdry_eff[i] + m->bdry_eff[j]);
            double F[3] = {0.0, 0.0, 0.0}, el;
            if (m->cci) {
                const double* xj = m->x + 3 * j;
                const double* uj = (m->bc[j] >= 0) ? m->U + 3 * j : us + 3 * j;
                double xv[3] = {xj[0] - xi[0], xj[1] - xi[1], xj[2] - xi[2]};
                double ev[3] = {uj[0] - ui[0], uj[1] - ui[1], uj[2] - ui[2]};
                bond_force(m, xv, ev, ecrit, spring, be, 2.0, F, &el);
                m->eed[i] += el;
            } else {
                for (int g = 0; g < m->npt; ++g) {
                    const double* q = m->xg + (j * m->npt + g) * 3;
                    const double* ugp = m->ug + (j * m->npt + g) * 3;
                    double xv[3] = {q[0] - xi[0], q[1] - xi[1], q[2] - xi[2]};
                    double ev[3] = {ugp[0] - ui[0], ugp[1] - ui[1], ugp[2] - ui[2]};
                    double w1 = m->gw[3 * g], w2 = m->gw[3 * g + 1], w3 = m->gw[3 * g + 2];
                    double effw = pow(w1 * w2 * w3, 1.0 / 3.0);
                    double fp[3];
                    bond_force(m, xv, ev, ecrit, spring, be, effw, fp, &el);
                    m->eed[i] += el;
                    F[0] += vol8 * w1 * w2 * w3 * fp[0];
                    F[1] += vol8 * w1 * w2 * w3 * fp[1];
                    F[2] += vol8 * w1 * w2 * w3 * fp[2];
                }
            }
            m->vbuf[3 * i + 0] += (F[0] + body[0]) * dts / rho;
            m->vbuf[3 * i + 1] += (F[1] + body[1]) * dts / rho;
            m->vbuf[3 * i + 2] += (F[2] + body[2]) * dts / rho;
        }
        /* project rule: a TRACTION boundary condition adds the body-force
         * density value*factor/dx once per stage on its nodes */
        int b = m->bc[i];
        if (b >= 0 && m->bc_type[b] == OR_TRACTION) {
            double fac = time_factor(m, b, t);
            for (int a = 0; a < 3; ++a)
                if (m->bc_dir[3 * b + a] == 1) {
                    double tb = m->bc_val[9 * b + a] * fac / m->dx;
                    m->vbuf[3 * i + a] += tb * dts / rho;
                }
        }
    }
    update_node_bc(m, t);
    for (int64_t i = 0; i < 3 * m->n; ++i) k[i] = m->vbuf[i] * dts;
}

void or_gather(or_model* m, double t, const double* us) {
    if (m->cci) return;
    int npt = m->npt;
    /* UpdateIntgPointStatusWithBC, pdDataManager.cpp:2604-2703 */
    for (int64_t i = 0; i < m->n; ++i) {
        int b = m->bc[i];
        if (b < 0) continue;
        int ty = m->bc_type[b];
        double fac = time_factor(m, b, t);
        const double* v = m->bc_val + 9 * b;
        for (int a = 0; a < 3; ++a) {
            if (m->bc_dir[3 * b + a] != 1) continue;
            for (int g = 0; g < npt; ++g) {
                double* o = m->ug + (i * npt + g) * 3;
                const double* q = m->xg + (i * npt + g) * 3;
                if (ty == OR_DISPL) o[a] = v[a] * fac;
                else if (ty == OR_DISPLGRAD) o[a] = (v[3 * a] * q[0] + v[3 * a + 1] * q[1] + v[3 * a + 2] * q[2]) * fac;
            }
        }
    }
    for (int64_t i = 0; i < m->n; ++i) {
        if (m->bc[i] >= 0) continue;
        if (m->mls) {
            int64_t nc = m->cb_ptr[i + 1] - m->cb_ptr[i];
            const int32_t* cb = m->cb_idx + m->cb_ptr[i];
            for (int g = 0; g < npt; ++g) {
                const double* c = m->coeff + m->cb_ptr[i] * npt + (int64_t)g * nc;
                double a1 = 0.0, a2 = 0.0, a3 = 0.0;
                for (int64_t k = 0; k < nc; ++k) {
                    const double* u = us + 3 * (int64_t)cb[k];
                    a1 += u[0] * c[k];
                    a2 += u[1] * c[k];
                    a3 += u[2] * c[k];
                }
                double* o = m->ug + (i * npt + g) * 3;
                o[0] = a1; o[1] = a2; o[2] = a3;
            }
        } else {
            double* o = m->ug + i * npt * 3;
            o[0] = us[3 * i]; o[1] = us[3 * i + 1]; o[2] = us[3 * i + 2];
        }
    }
}

static void record_stage(const or_model* m, const double* us, double* out) {
    int64_t n3 = 3 * m->n;
    memcpy(out, m->U, sizeof(double) * (size_t)n3);
    memcpy(out + n3, us, sizeof(double) * (size_t)n3);
    memcpy(out + 2 * n3, m->ug, sizeof(double) * (size_t)(n3 * m->npt));
}

/* One RK4 step.  With tape != NULL, the inputs of the four force stages
 * (U, trial displacement, Gauss-point displacements: 3n + 3n + 3n*npt
 * values each) are copied there before each stage. */
static void rk4_step_taped(or_model* m, double dt, double t, double* tape) {
    int64_t n3 = 3 * m->n;
    int64_t per = 2 * n3 + n3 * m->npt;
    /* InitDynamicSolve, pdDataManager2.cpp:410-439 */
    for (int64_t i = 0; i < n3; ++i) m->vbuf[i] = m->V[i];
    for (int64_t i = 0; i < m->n; ++i) m->eed[i] = 0.0;
    double* u1 = (double*)malloc(sizeof(double) * (size_t)n3 * 6);
    double *u234 = u1 + n3, *k1 = u1 + 2 * n3, *k24 = u1 + 3 * n3, *k3 = u1 + 4 * n3, *k4 = u1 + 5 * n3;
    double dtHalf = 0.5 * dt, dt6 = 1.0 / 6.0;
    memcpy(u1, m->U, sizeof(double) * (size_t)n3);
    if (tape) record_stage(m, u1, tape + 0 * per);
    or_force_stage(m, dtHalf, t, u1, k1);
    for (int64_t i = 0; i < n3; ++i) u234[i] = u1[i] + 0.5 * k1[i];
    or_gather(m, t, u234);
    if (tape) record_stage(m, u234, tape + 1 * per);
    or_force_stage(m, dtHalf, t, u234, k24);
    for (int64_t i = 0; i < n3; ++i) u234[i] = u1[i] + 0.5 * k24[i];
    or_gather(m, t, u234);
    if (tape) record_stage(m, u234, tape + 2 * per);
    or_force_stage(m, dt, t, u234, k3);
    for (int64_t i = 0; i < n3; ++i) { u234[i] = u1[i] + k3[i]; k3[i] += k24[i]; }
    or_gather(m, t, u234);
    if (tape) record_stage(m, u234, tape + 3 * per);
    or_force_stage(m, dt, t, u234, k4);
    for (int64_t i = 0; i < m->n; ++i) {
        double rho = m->mat_density[m->mat[i]];
        for (int a = 0; a < 3; ++a) {
            int64_t r = 3 * i + a;
            double u = m->U[r];
            if (m->bc[i] >= 0) m->U[r] = u + dt6 * (k1[r] + k4[r] + 2.0 * k3[r]);
            else m->U[r] = u + dt6 * (k1[r] + k4[r] + 2.0 * k3[r]) - dt * m->damping * m->V[r] * dt / rho;
        }
        for (int a = 0; a < 3; ++a) m->vbuf[3 * i + a] += -m->damping * m->V[3 * i + a] * dt / rho;
        for (int a = 0; a < 3; ++a) m->V[3 * i + a] = m->vbuf[3 * i + a];
    }
    double ke = 0.0, ee = 0.0, vol = pow(m->dx, 3.0);
    for (int64_t i = 0; i < m->n; ++i) {
        double rho = m->mat_density[m->mat[i]];
        const double* v = m->V + 3 * i;
        double velsq = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        ee += vol * m->eed[i];
        ke += 0.5 * rho * velsq * vol;
    }
    m->ke = ke;
    m->ee = ee;
    or_gather(m, t, m->U);
    free(u1);
}

void or_rk4_step(or_model* m, double dt, double t) { rk4_step_taped(m, dt, t, NULL); }

/* ------------------------------------------------------------ AI form -- */

/* pd_ai_region's layout (pdmtel_b200.h) */
typedef struct {
    double a, b;
    uint8_t axis[3];
    uint8_t lim[4];
    uint8_t flags;
} or_ai_region;

typedef struct {
    or_model* m;
    int trap;
    double xj[3];               /* node j in the family coordinates of node i */
    int64_t i, j;
    const double* ui;
    double ecrit, spring, be, t;
    const double* us;
    const double* tab;          /* node j's coefficient list */
    int64_t ncb;
    const int32_t* cb;
    const or_ai_region* R;
    int counter;                /* _intgPointCounter */
    int failed;
} ai_state;

/* SolveBinaryQuadric with its centre at the origin (pdIntgManager2.cpp:812-834) */
static double ai_quadric(double r_sq, double xy) {
    double v = r_sq - (xy - 0.0) * (xy - 0.0);
    if (v < 0.0) return -1.0;
    return sqrt(v);
}

/* middle-direction limits (pdIntgManager2.cpp:440-617) */
static double ai_ylimit(const ai_state* s, int code, double x) {
    const double dx = s->m->dx, delta = s->m->delta;
    if (code < 8) {
        int ax = code / 2;
        return (code % 2) ? s->xj[ax] + 0.5 * dx : s->xj[ax] - 0.5 * dx;
    }
    int c = code - 8;
    int pos = c % 2, high = (c / 2) % 2, solved = (c / 4) / 3, arg = (c / 4) % 3;
    int third = 3 - solved - arg;
    double plane = high ? s->xj[third] + 0.5 * dx : s->xj[third] - 0.5 * dx;
    double v = ai_quadric(delta * delta - plane * plane, x);
    if (v < 0.0) v = 0.0;
    return pos ? v : -v;
}

/* inner-direction limits (pdIntgManager2.cpp:622-682) */
static double ai_zlimit(const ai_state* s, int code, double x, double y) {
    const double dx = s->m->dx, delta = s->m->delta;
    if (code < 8) {
        int ax = code / 2;
        return (code % 2) ? s->xj[ax] + 0.5 * dx : s->xj[ax] - 0.5 * dx;
    }
    double sq = delta * delta - x * x - y * y;
    double v = (sq < 0.0) ? 0.0 : sqrt(sq);
    return (code % 2) ? v : -v;
}

/* the integrand CalcBondBasedForce (pdIntgManager2.cpp:92-310) at the local
 * point (x1, x2, x3) */
static void ai_integrand(ai_state* s, double x1, double x2, double x3, double* f) {
    or_model* m = s->m;
    double xi1 = x1 - 0.0, xi2 = x2 - 0.0, xi3 = x3 - 0.0;
    double eta[3];
    int b = m->bc[s->j];
    if (m->mls) {
        double u[3] = {0.0, 0.0, 0.0};
        /* the MLS value; a boundary-condition node overrides its prescribed directions */
        const double* c = s->tab + (int64_t)s->counter * s->ncb;
        for (int64_t q = 0; q < s->ncb; ++q) {
            const double* d = s->us + 3 * (int64_t)s->cb[q];
            u[0] += d[0] * c[q];
            u[1] += d[1] * c[q];
            u[2] += d[2] * c[q];
        }
        if (b >= 0) {
            double fac = time_factor(m, b, s->t);
            const int32_t* dir = m->bc_dir + 3 * b;
            const double* v = m->bc_val + 9 * b;
            const double* X = m->x + 3 * s->i;
            double xg[3] = {x1 + X[0], x2 + X[1], x3 + X[2]};
            for (int a = 0; a < 3; ++a) {
                if (dir[a] != 1) continue;
                if (m->bc_type[b] == OR_DISPL) u[a] = v[a] * fac;
                else if (m->bc_type[b] == OR_DISPLGRAD)
                    u[a] = (v[3 * a] * xg[0] + v[3 * a + 1] * xg[1] + v[3 * a + 2] * xg[2]) * fac;
            }
        }
        eta[0] = u[0] - s->ui[0];
        eta[1] = u[1] - s->ui[1];
        eta[2] = u[2] - s->ui[2];
    } else {
        const double* v = m->bc_val + 9 * b;
        for (int a = 0; a < 3; ++a) eta[a] = v[3 * a] * xi1 + v[3 * a + 1] * xi2 + v[3 * a + 2] * xi3;
    }
    double r = sqrt(xi1 * xi1 + xi2 * xi2 + xi3 * xi3);
    double y1 = xi1 + eta[0], y2 = xi2 + eta[1], y3 = xi3 + eta[2];
    double p = sqrt(y1 * y1 + y2 * y2 + y3 * y3);
    double beta = 1.0;
    double u = p - r;
    double stretch = u / r;
    if (u <= 0.0 || (u > 0.0 && stretch <= s->ecrit)) {
        f[0] = s->be * beta * s->spring * stretch * (xi1 + eta[0]) / p;
        f[1] = s->be * beta * s->spring * stretch * (xi2 + eta[1]) / p;
        f[2] = s->be * beta * s->spring * stretch * (xi3 + eta[2]) / p;
        m->eed[s->i] += s->be * 0.5 * (0.5 * beta * (s->spring / r) * u * u);
    } else {
        f[0] = f[1] = f[2] = 0.0;
        s->failed += 1;
    }
}

static void ai_x1(ai_state* s, double x, double* f);
static void ai_x2(ai_state* s, double x, double y, double* f);

/* CalcIntgX3 (pdIntgManager.cpp:282-345): the point in x, y, z order */
static void ai_x3(ai_state* s, double x, double y, double z, double* f) {
    double p[3];
    p[s->R->axis[0]] = x;
    p[s->R->axis[1]] = y;
    p[s->R->axis[2]] = z;
    ai_integrand(s, p[0], p[1], p[2], f);
    ++s->counter;
}

static void ai_eval(ai_state* s, int level, double v, double x, double y, double* f) {
    if (level == 1) ai_x1(s, v, f);
    else if (level == 2) ai_x2(s, x, v, f);
    else ai_x3(s, x, y, v, f);
}

/* CalcTrapzdQuad, cases 1-3 (pdIntgManager.cpp:347-451) */
static void ai_trapz(ai_state* s, int level, double a, double b, double x, double y, double* out) {
    double f1[3], f2[3], f3[3], f4[3], f5[3];
    if (s->trap == 1) {
        ai_eval(s, level, a, x, y, f1);
        ai_eval(s, level, b, x, y, f2);
        for (int c = 0; c < 3; ++c) out[c] = (b - a) * (0.5 * f1[c] + 0.5 * f2[c]);
    } else if (s->trap == 2) {
        ai_eval(s, level, a, x, y, f1);
        ai_eval(s, level, 0.5 * (a + b), x, y, f2);
        ai_eval(s, level, b, x, y, f3);
        for (int c = 0; c < 3; ++c) out[c] = 0.5 * (b - a) * (0.5 * f1[c] + f2[c] + 0.5 * f3[c]);
    } else {
        ai_eval(s, level, a, x, y, f1);
        ai_eval(s, level, 0.25 * (3.0 * a + b), x, y, f2);
        ai_eval(s, level, 0.5 * (a + b), x, y, f3);
        ai_eval(s, level, 0.25 * (a + 3.0 * b), x, y, f4);
        ai_eval(s, level, b, x, y, f5);
        for (int c = 0; c < 3; ++c)
            out[c] = 0.25 * (b - a) * (0.5 * f1[c] + f2[c] + f3[c] + f4[c] + 0.5 * f5[c]);
    }
}

/* CalcIntgX1 (pdIntgManager.cpp:130-204) */
static void ai_x1(ai_state* s, double x, double* f) {
    double a = ai_ylimit(s, s->R->lim[0], x), b = ai_ylimit(s, s->R->lim[1], x);
    if (fabs(a - b) <= 1.0e-10) { f[0] = f[1] = f[2] = 0.0; return; }
    ai_trapz(s, 2, a, b, x, 0.0, f);
}

/* CalcIntgX2 (pdIntgManager.cpp:206-280) */
static void ai_x2(ai_state* s, double x, double y, double* f) {
    double a = ai_zlimit(s, s->R->lim[2], x, y), b = ai_zlimit(s, s->R->lim[3], x, y);
    if (fabs(a - b) <= 1.0e-10) { f[0] = f[1] = f[2] = 0.0; return; }
    ai_trapz(s, 3, a, b, x, y, f);
}

/* CalcIntg3D (pdIntgManager.cpp:49-128) over one region */
static void ai_region3d(ai_state* s, const or_ai_region* R, double* f) {
    s->R = R;
    s->counter = 0;
    if (fabs(R->a - R->b) <= 1.0e-10) { f[0] = f[1] = f[2] = 0.0; return; }
    ai_trapz(s, 1, R->a, R->b, 0.0, 0.0, f);
}

static int64_t ai_entry(const or_model* m, int64_t i, int64_t j) {
    int64_t lo = m->fam_ptr[i], hi = m->fam_ptr[i + 1];
    while (lo < hi) {
        int64_t mid = lo + (hi - lo) / 2;
        if (m->fam_col[mid] < j) lo = mid + 1;
        else hi = mid;
    }
    return (lo < m->fam_ptr[i + 1] && m->fam_col[lo] == j) ? lo : -1;
}

void or_ai_force_stage(or_model* m, int trap, const int64_t* reg_ptr, const void* regs, const int64_t* tab_ptr,
                       const double* tab_coeff, uint8_t* ai_broken, int32_t* dmg, double dts, double t,
                       const double* us, double* k) {
    const or_ai_region* RG = (const or_ai_region*)regs;
    for (int64_t i = 0; i < m->n; ++i) {
        int mi = m->mat[i];
        double rho = m->mat_density[mi];
        double body[3] = {m->mat_grav[3 * mi] * rho, m->mat_grav[3 * mi + 1] * rho, m->mat_grav[3 * mi + 2] * rho};
        const double* ui = (m->bc[i] >= 0) ? m->U + 3 * i : us + 3 * i;
        for (int64_t p = m->fam_ptr[i]; p < m->fam_ptr[i + 1]; ++p) {
            if (ai_broken[p]) continue;
            int64_t j = m->fam_col[p];
            int mj = m->mat[j];
            ai_state s;
            memset(&s, 0, sizeof(s));
            s.m = m;
            s.trap = trap;
            for (int a = 0; a < 3; ++a) s.xj[a] = m->x[3 * j + a] - m->x[3 * i + a];
            s.i = i;
            s.j = j;
            s.ui = ui;
            s.ecrit = (m->mat_ecrit[mj] < m->mat_ecrit[mi]) ? m->mat_ecrit[mj] : m->mat_ecrit[mi];
            s.spring = pair_spring(m, i, j);
            s.be = 0.5 * (m->bdry_eff[i] + m->bdry_eff[j]);
            s.t = t;
            s.us = us;
            if (m->mls) {
                s.ncb = m->cb_ptr[j + 1] - m->cb_ptr[j];
                s.cb = m->cb_idx + m->cb_ptr[j];
                int64_t off = 0;
                for (int64_t q = 0; q < j; ++q) off += (tab_ptr[q + 1] - tab_ptr[q]) * (m->cb_ptr[q + 1] - m->cb_ptr[q]);
                s.tab = tab_coeff + off;
            }
            double F[3] = {0.0, 0.0, 0.0};
            int64_t r0 = reg_ptr[p], r1 = reg_ptr[p + 1];
            if (r1 > r0 && (RG[r0].flags & 1)) {
                ai_region3d(&s, &RG[r0], F);
            } else {
                for (int64_t r = r0; r < r1; ++r) {
                    double st[3];
                    ai_region3d(&s, &RG[r], st);
                    F[0] += st[0];
                    F[1] += st[1];
                    F[2] += st[2];
                }
            }
            if (s.failed) {
                int64_t q = ai_entry(m, j, i);
                ai_broken[p] = 1;
                if (q >= 0) ai_broken[q] = 1;
                dmg[i] += s.failed;
            }
            m->vbuf[3 * i + 0] += (F[0] + body[0]) * dts / rho;
            m->vbuf[3 * i + 1] += (F[1] + body[1]) * dts / rho;
            m->vbuf[3 * i + 2] += (F[2] + body[2]) * dts / rho;
        }
        int b = m->bc[i];
        if (b >= 0 && m->bc_type[b] == OR_TRACTION) {
            double fac = time_factor(m, b, t);
            for (int a = 0; a < 3; ++a)
                if (m->bc_dir[3 * b + a] == 1) {
                    double tb = m->bc_val[9 * b + a] * fac / m->dx;
                    m->vbuf[3 * i + a] += tb * dts / rho;
                }
        }
    }
    update_node_bc(m, t);
    for (int64_t i = 0; i < 3 * m->n; ++i) k[i] = m->vbuf[i] * dts;
}

/* ------------------------------------------------------------ adjoint -- */

/* Project rule, no counterpart in the reference: reverse accumulation of
 * dJ/d(spring factor) through rk4_step_taped.  One Gauss point's force is
 * f = be*beta*c*s*y/p with s = (p-r)/r (bond_force), i.e. k (1/r - 1/p) y
 * with k = be*beta*c*W, whose Jacobian in y is k [(1/r - 1/p) I + y y^T/p^3];
 * a point past the critical stretch has f = 0 and no derivative. */

/* the stage's BC overwrite sets U (DISPL, DISPLGRAD) or vbuf (also VELOC) */
static int fixes_u(const or_model* m, int64_t i, int a) {
    int b = m->bc[i];
    if (b < 0 || m->bc_dir[3 * b + a] != 1) return 0;
    return m->bc_type[b] == OR_DISPL || m->bc_type[b] == OR_DISPLGRAD;
}
static int fixes_v(const or_model* m, int64_t i, int a) {
    int b = m->bc[i];
    if (b < 0 || m->bc_dir[3 * b + a] != 1) return 0;
    return m->bc_type[b] != OR_TRACTION;
}
/* a Gauss-point entry of a BC node that the gather prescribes */
static int gather_sets(const or_model* m, int64_t i, int a) { return fixes_u(m, i, a); }

/* VJP of the bond forces of one stage.  lam [n][3]: adjoint of each node's
 * summed force.  Adds to bown (the node's own displacement as read), bug
 * (Gauss-point displacements) and gradf. */
static void force_vjp(const or_model* m, const double* Us, const double* us, const double* ug, const double* lam,
                      double* bown, double* bug, double* gradf) {
    double vol8 = pow(m->dx, 3) / 8.0;
    for (int64_t i = 0; i < m->n; ++i) {
        const double* ui = (m->bc[i] >= 0) ? Us + 3 * i : us + 3 * i;
        const double* xi = m->x + 3 * i;
        const double* l = lam + 3 * i;
        for (int64_t p = m->fam_ptr[i]; p < m->fam_ptr[i + 1]; ++p) {
            if (m->broken && m->broken[p]) continue;
            int64_t j = m->fam_col[p];
            int mi = m->mat[i], mj = m->mat[j];
            double ecrit = dmin2(m->mat_ecrit[mi], m->mat_ecrit[mj]);
            double cmin = dmin2(m->mat_spring[mi], m->mat_spring[mj]);
            double c = pair_spring(m, i, j);
            double be = 0.5 * (m->bdry_eff[i] + m->bdry_eff[j]);
            double dc = 0.0; /* dJ/dc_ij */
            for (int g = 0; g < m->npt; ++g) {
                const double* q = m->xg + (j * m->npt + g) * 3;
                const double* ugp = ug + (j * m->npt + g) * 3;
                double w1 = m->gw[3 * g], w2 = m->gw[3 * g + 1], w3 = m->gw[3 * g + 2];
                double W = vol8 * w1 * w2 * w3;
                double effw = pow(w1 * w2 * w3, 1.0 / 3.0);
                double xv[3], ev[3], y[3], qq = 0.0;
                for (int a = 0; a < 3; ++a) {
                    xv[a] = q[a] - xi[a];
                    ev[a] = ugp[a] - ui[a];
                    y[a] = xv[a] + ev[a];
                    qq += ev[a] * (2.0 * xv[a] + ev[a]);
                }
                double r = sqrt(xv[0] * xv[0] + xv[1] * xv[1] + xv[2] * xv[2]);
                double pl = sqrt(y[0] * y[0] + y[1] * y[1] + y[2] * y[2]);
                double ext = qq / (pl + r); /* p - r without cancellation */
                if (ext > 0.0 && ext / r > ecrit) continue;
                double beta = beta_factor(r, m->delta, effw * m->dx / 2.0, 0, 0);
                double a0 = ext / (r * pl); /* 1/r - 1/p */
                double yl = y[0] * l[0] + y[1] * l[1] + y[2] * l[2];
                double kk = be * beta * c * W;
                for (int a = 0; a < 3; ++a) {
                    double dy = kk * (a0 * l[a] + y[a] * yl / (pl * pl * pl));
                    bown[3 * i + a] -= dy;
                    bug[(j * m->npt + g) * 3 + a] += dy;
                }
                dc += be * beta * W * a0 * yl;
            }
            if (m->spring_factor) {
                gradf[i] += 0.5 * cmin * dc;
                gradf[j] += 0.5 * cmin * dc;
            }
        }
    }
}

/* transpose of or_gather's node rows: bus[contributor] += coeff * bug */
static void gather_t(const or_model* m, const double* bug, double* bus) {
    int npt = m->npt;
    for (int64_t i = 0; i < m->n; ++i) {
        if (m->bc[i] >= 0) continue;
        if (m->mls) {
            int64_t nc = m->cb_ptr[i + 1] - m->cb_ptr[i];
            const int32_t* cb = m->cb_idx + m->cb_ptr[i];
            for (int g = 0; g < npt; ++g) {
                const double* c = m->coeff + m->cb_ptr[i] * npt + (int64_t)g * nc;
                const double* b = bug + (i * npt + g) * 3;
                for (int64_t k = 0; k < nc; ++k)
                    for (int a = 0; a < 3; ++a) bus[3 * (int64_t)cb[k] + a] += c[k] * b[a];
            }
        } else {
            for (int a = 0; a < 3; ++a) bus[3 * i + a] += bug[i * npt * 3 + a];
        }
    }
}

/* move the BC nodes' carried Gauss-point entries of bug into carry */
static void carry_bc_entries(const or_model* m, const double* bug, double* carry) {
    for (int64_t i = 0; i < m->n; ++i) {
        if (m->bc[i] < 0) continue;
        for (int g = 0; g < m->npt; ++g)
            for (int a = 0; a < 3; ++a)
                if (!gather_sets(m, i, a)) carry[(i * m->npt + g) * 3 + a] += bug[(i * m->npt + g) * 3 + a];
    }
}

/* reverse of one step; bU, bV, bug: adjoints of the step's output state in,
 * of its input state out */
static void rk4_step_reverse(const or_model* m, double dt, const double* tape, double* bU, double* bV, double* bug,
                             double* w) {
    int64_t n = m->n, n3 = 3 * n, ng = n3 * m->npt, per = 2 * n3 + ng;
    double *bk[5], *bvb, *bu1, *bUs, *bown, *bus, *lam, *bugs, *carry;
    bk[0] = NULL;
    for (int s = 1; s <= 4; ++s) bk[s] = w + (s - 1) * n3;
    bvb = w + 4 * n3; bu1 = w + 5 * n3; bUs = w + 6 * n3; bown = w + 7 * n3; bus = w + 8 * n3; lam = w + 9 * n3;
    bugs = w + 10 * n3; carry = bugs + ng;
    memset(w, 0, sizeof(double) * (size_t)(10 * n3 + 2 * ng));
    /* final gather: ug_end = G(U_new) on free nodes, carried on BC nodes */
    gather_t(m, bug, bU);
    carry_bc_entries(m, bug, carry);
    /* combination and damping */
    for (int64_t i = 0; i < n; ++i) {
        double rho = m->mat_density[m->mat[i]];
        for (int a = 0; a < 3; ++a) {
            int64_t r = 3 * i + a;
            double g = bU[r];
            bk[1][r] = g / 6.0;
            bk[4][r] = g / 6.0;
            bk[3][r] = g / 3.0; /* k3 (after k3 += k24) enters twice */
            bk[2][r] = g / 3.0;
            bUs[r] = g;
            double v = -m->damping * dt / rho * bV[r];
            if (m->bc[i] < 0) v += -dt * m->damping * dt / rho * g;
            bvb[r] = bV[r];
            bV[r] = v;
        }
    }
    for (int s = 4; s >= 1; --s) {
        double dts = s >= 3 ? dt : 0.5 * dt;
        const double* T = tape + (s - 1) * per;
        for (int64_t r = 0; r < n3; ++r) bvb[r] += dts * bk[s][r];
        for (int64_t i = 0; i < n; ++i)
            for (int a = 0; a < 3; ++a) {
                if (fixes_v(m, i, a)) bvb[3 * i + a] = 0.0;
                if (fixes_u(m, i, a)) bUs[3 * i + a] = 0.0;
            }
        for (int64_t i = 0; i < n; ++i) {
            double rho = m->mat_density[m->mat[i]];
            for (int a = 0; a < 3; ++a) lam[3 * i + a] = bvb[3 * i + a] * dts / rho;
        }
        memset(bown, 0, sizeof(double) * (size_t)n3);
        memset(bugs, 0, sizeof(double) * (size_t)ng);
        force_vjp(m, T, T + n3, T + 2 * n3, lam, bown, bugs, w + 10 * n3 + 2 * ng);
        memset(bus, 0, sizeof(double) * (size_t)n3);
        for (int64_t i = 0; i < n; ++i)
            for (int a = 0; a < 3; ++a) {
                if (m->bc[i] >= 0) bUs[3 * i + a] += bown[3 * i + a];
                else bus[3 * i + a] = bown[3 * i + a];
            }
        carry_bc_entries(m, bugs, carry);
        if (s >= 2) {
            gather_t(m, bugs, bus);
            double alpha = s == 4 ? 1.0 : 0.5;
            for (int64_t r = 0; r < n3; ++r) {
                bu1[r] += bus[r];
                bk[s - 1][r] += alpha * bus[r];
            }
        } else {
            for (int64_t r = 0; r < n3; ++r) bu1[r] += bus[r];
            /* ug at stage 1 is the step's input: free nodes' rows */
            for (int64_t i = 0; i < n; ++i) {
                double* o = bug + i * m->npt * 3;
                const double* src = (m->bc[i] >= 0) ? carry + i * m->npt * 3 : bugs + i * m->npt * 3;
                for (int e = 0; e < m->npt * 3; ++e) o[e] = src[e];
            }
        }
    }
    for (int64_t r = 0; r < n3; ++r) {
        bU[r] = bUs[r] + bu1[r];
        bV[r] += bvb[r];
    }
}

int or_adjoint_grad(or_model* m, double dt, double t0, int nsteps, const double* lamU, const double* lamV,
                    double* gradf) {
    int64_t n = m->n, n3 = 3 * n, ng = n3 * m->npt, per = 2 * n3 + ng;
    double* tape = (double*)malloc(sizeof(double) * (size_t)(4 * per) * (size_t)nsteps);
    double* w = (double*)malloc(sizeof(double) * (size_t)(10 * n3 + 2 * ng + n));
    double* st = (double*)malloc(sizeof(double) * (size_t)(2 * n3 + ng));
    if (!tape || !w || !st) {
        free(tape); free(w); free(st);
        return -1;
    }
    double t = t0;
    for (int k = 0; k < nsteps; ++k) {
        t += dt;
        rk4_step_taped(m, dt, t, tape + (int64_t)k * 4 * per);
    }
    double *bU = st, *bV = st + n3, *bug = st + 2 * n3;
    for (int64_t r = 0; r < n3; ++r) {
        bU[r] = lamU[r];
        bV[r] = lamV ? lamV[r] : 0.0;
    }
    memset(bug, 0, sizeof(double) * (size_t)ng);
    double* gacc = w + 10 * n3 + 2 * ng;
    memset(gacc, 0, sizeof(double) * (size_t)n);
    for (int k = nsteps - 1; k >= 0; --k) {
        /* rk4_step_reverse clears w except the gradient that follows it */
        rk4_step_reverse(m, dt, tape + (int64_t)k * 4 * per, bU, bV, bug, w);
    }
    for (int64_t i = 0; i < n; ++i) gradf[i] = gacc[i];
    free(tape); free(w); free(st);
    return 0;
}

/* ------------------------------------------------- boundary effect ----- */

static double bdry_type_one(const or_model* m, int mi, double h) {
    double full = 3.0 * m->mat_ymod[mi];
    double part = full - 0.5 * m->mat_spring[mi] * OR_PI *
                             (pow(m->delta, 4) / 4.0 - h * pow(m->delta, 3) / 3.0 + pow(h, 4) / 12.0);
    return full / part;
}

static double bdry_general(const or_model* m, int64_t i) {
    double e11 = 1.0e-4;
    int mi = m->mat[i];
    double ecrit = m->mat_ecrit[mi], spring = m->mat_spring[mi];
    const double* X = m->x + 3 * i;
    double eps[9] = {e11, 0.0, 0.0, 0.0, e11, 0.0, 0.0, 0.0, e11};
    double sum = 0.0;
    double volj = pow(m->dx, 3.0);
    for (int64_t p = m->fam_ptr[i]; p < m->fam_ptr[i + 1]; ++p) {
        if (m->broken && m->broken[p]) continue;
        const double* Y = m->x + 3 * (int64_t)m->fam_col[p];
        double xi1 = Y[0] - X[0], xi2 = Y[1] - X[1], xi3 = Y[2] - X[2];
        double e1 = eps[0] * xi1 + eps[1] * xi2 + eps[2] * xi3;
        double e2 = eps[3] * xi1 + eps[4] * xi2 + eps[5] * xi3;
        double e3 = eps[6] * xi1 + eps[7] * xi2 + eps[8] * xi3;
        double r = sqrt(xi1 * xi1 + xi2 * xi2 + xi3 * xi3);
        double p1 = xi1 + e1, p2 = xi2 + e2, p3 = xi3 + e3;
        double pp = sqrt(p1 * p1 + p2 * p2 + p3 * p3);
        double u = pp - r, s = u / r, el;
        if (u <= 0 || (u > 0 && s <= ecrit)) el = 0.5 * (spring / r) * u * u;
        else el = 0.0;
        double beta = beta_factor(r, m->delta, m->dx, m->cci, m->cci_mdf);
        double elj = el * beta * volj;
        sum += 0.5 * elj;
    }
    double pinf = 3.0 * m->mat_ymod[mi] * e11 * e11;
    return pinf / sum;
}

int or_bdry_eff(const or_model* m, const int* dims, const double* center, double* bE) {
    double dx = m->dx, delta = m->delta, tol = 1.0e-4 * dx;
    int vd = 2 * ((int)(delta / dx) + 1);
    double o[3] = {0.0, 0.0, 0.0};
    int full = 0;
    for (int nn = 1; nn != vd + 1; ++nn)
        for (int mm = 1; mm != vd + 1; ++mm)
            for (int l = 1; l != vd + 1; ++l) {
                double q[3] = {(l - vd * 0.5) * dx, (mm - vd * 0.5) * dx, (nn - vd * 0.5) * dx};
                double mn, mx;
                dist_to_cube(o, q, dx, &mn, &mx);
                if (mn < delta + tol) ++full;
            }
    double x1lo = -dims[0] * 0.5 * dx + center[0], x1hi = dims[0] * 0.5 * dx + center[0];
    double x2lo = -dims[1] * 0.5 * dx + center[1], x2hi = dims[1] * 0.5 * dx + center[1];
    double x3lo = -dims[2] * 0.5 * dx + center[2], x3hi = dims[2] * 0.5 * dx + center[2];
    double ns = ((int)(delta / dx)) * dx;
    for (int64_t i = 0; i < m->n; ++i) {
        double a = m->x[3 * i], b = m->x[3 * i + 1], c = m->x[3 * i + 2];
        int mi = m->mat[i];
        if (m->fam_ptr[i + 1] - m->fam_ptr[i] == full) bE[i] = 1.0;
        else if (a >= x1hi - ns && a <= x1hi && b >= x2lo + ns && b <= x2hi - ns && c >= x3lo + ns && c <= x3hi - ns)
            bE[i] = bdry_type_one(m, mi, x1hi - a);
        else if (a >= x1lo && a <= x1lo + ns && b >= x2lo + ns && b <= x2hi - ns && c >= x3lo + ns && c <= x3hi - ns)
            bE[i] = bdry_type_one(m, mi, a - x1lo);
        else if (b >= x2hi - ns && b <= x2hi && a >= x1lo + ns && a <= x1hi - ns && c >= x3lo + ns && c <= x3hi - ns)
            bE[i] = bdry_type_one(m, mi, x2hi - b);
        else if (b >= x2lo && b <= x2lo + ns && a >= x1lo + ns && a <= x1hi - ns && c >= x3lo + ns && c <= x3hi - ns)
            bE[i] = bdry_type_one(m, mi, b - x2lo);
        else if (c >= x3hi - ns && c <= x3hi && a >= x1lo + ns && a <= x1hi - ns && b >= x2lo + ns && b <= x2hi - ns)
            bE[i] = bdry_type_one(m, mi, x3hi - c);
        else if (c >= x3lo && c <= x3lo + ns && a >= x1lo + ns && a <= x1hi - ns && b >= x2lo + ns && b <= x2hi - ns)
            bE[i] = bdry_type_one(m, mi, c - x3lo);
        else
            bE[i] = bdry_general(m, i);
    }
    return full;
}

/* ----------------------------------------------------------- static ---- */

/* prescribed value of dof (i,a) in the static system, pdSolve.cpp:215-262;
 * returns 0 for a free dof */
static int static_prescribed(const or_model* m, int64_t i, int a, double t, double* val) {
    int b = m->bc[i];
    if (b < 0 || m->bc_dir[3 * b + a] != 1) return 0;
    if (m->bc_type[b] == OR_DISPL) { *val = m->bc_val[9 * b + a]; return 1; }
    if (m->bc_type[b] == OR_VELOC) { *val = m->bc_val[9 * b + a] * t; return 1; }
    return 0;
}

/* K restricted to free rows and free columns, applied to x (prescribed
 * entries of x are ignored); prescribed rows return x. */
void or_static_apply(const or_model* m, double t, const double* x, double* y) {
    double vol = pow(m->dx, 3.0), dummy;
    for (int64_t i = 0; i < m->n; ++i) {
        const double* X = m->x + 3 * i;
        int fi[3];
        for (int a = 0; a < 3; ++a) fi[a] = !static_prescribed(m, i, a, t, &dummy);
        double acc[3] = {0.0, 0.0, 0.0};
        for (int64_t p = m->fam_ptr[i]; p < m->fam_ptr[i + 1]; ++p) {
            if (m->broken && m->broken[p]) continue;
            int64_t j = m->fam_col[p];
            const double* Y = m->x + 3 * j;
            double xi[3] = {Y[0] - X[0], Y[1] - X[1], Y[2] - X[2]};
            double r = sqrt(xi[0] * xi[0] + xi[1] * xi[1] + xi[2] * xi[2]);
            double c = pair_spring(m, i, j);
            double r3 = pow(r, 3.0);
            int fj[3];
            for (int b = 0; b < 3; ++b) fj[b] = !static_prescribed(m, j, b, t, &dummy);
            for (int a = 0; a < 3; ++a) {
                for (int b = 0; b < 3; ++b) {
                    double cab = c * xi[a] * xi[b] / r3 * vol;
                    double d = (fi[b] ? x[3 * i + b] : 0.0) - (fj[b] ? x[3 * j + b] : 0.0);
                    acc[a] += cab * d;
                }
            }
        }
        for (int a = 0; a < 3; ++a) y[3 * i + a] = fi[a] ? acc[a] : x[3 * i + a];
    }
}

void or_static_rhs(const or_model* m, double t, double* bvec) {
    double vol = pow(m->dx, 3.0);
    for (int64_t i = 0; i < m->n; ++i) {
        const double* X = m->x + 3 * i;
        double pv[3];
        int fi[3];
        for (int a = 0; a < 3; ++a) { pv[a] = 0.0; fi[a] = !static_prescribed(m, i, a, t, &pv[a]); }
        double acc[3] = {0.0, 0.0, 0.0};
        for (int64_t p = m->fam_ptr[i]; p < m->fam_ptr[i + 1]; ++p) {
            if (m->broken && m->broken[p]) continue;
            int64_t j = m->fam_col[p];
            const double* Y = m->x + 3 * j;
            double xi[3] = {Y[0] - X[0], Y[1] - X[1], Y[2] - X[2]};
            double r = sqrt(xi[0] * xi[0] + xi[1] * xi[1] + xi[2] * xi[2]);
            double c = pair_spring(m, i, j);
            double r3 = pow(r, 3.0);
            double qv[3];
            int fj[3];
            for (int b = 0; b < 3; ++b) { qv[b] = 0.0; fj[b] = !static_prescribed(m, j, b, t, &qv[b]); }
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) {
                    double cab = c * xi[a] * xi[b] / r3 * vol;
                    if (!fi[b]) acc[a] -= cab * pv[b];
                    if (!fj[b]) acc[a] += cab * qv[b];
                }
        }
        int b = m->bc[i];
        for (int a = 0; a < 3; ++a) {
            if (!fi[a]) { bvec[3 * i + a] = pv[a]; continue; }
            double load = acc[a];
            if (b >= 0 && m->bc_type[b] == OR_TRACTION && m->bc_dir[3 * b + a] == 1)
                load += m->bc_val[9 * b + a] * time_factor(m, b, t) / m->dx;
            bvec[3 * i + a] = load;
        }
    }
}

int or_static_cg(const or_model* m, double t, const double* b, double* x, double rtol, int maxit, double* relres) {
    int64_t n3 = 3 * m->n;
    double* r = (double*)malloc(sizeof(double) * (size_t)n3 * 3);
    double *p = r + n3, *q = r + 2 * n3;
    or_static_apply(m, t, x, q);
    double bn = 0.0, rr = 0.0;
    for (int64_t i = 0; i < n3; ++i) { r[i] = b[i] - q[i]; p[i] = r[i]; bn += b[i] * b[i]; rr += r[i] * r[i]; }
    bn = sqrt(bn);
    if (bn == 0.0) bn = 1.0;
    int it = 0;
    while (sqrt(rr) / bn > rtol && it < maxit) {
        or_static_apply(m, t, p, q);
        double pq = 0.0;
        for (int64_t i = 0; i < n3; ++i) pq += p[i] * q[i];
        double alpha = rr / pq, rr2 = 0.0;
        for (int64_t i = 0; i < n3; ++i) { x[i] += alpha * p[i]; r[i] -= alpha * q[i]; rr2 += r[i] * r[i]; }
        double beta = rr2 / rr;
        for (int64_t i = 0; i < n3; ++i) p[i] = r[i] + beta * p[i];
        rr = rr2;
        ++it;
    }
    if (relres) *relres = sqrt(rr) / bn;
    free(r);
    return (sqrt(rr) / bn <= rtol) ? it : -1;
}
