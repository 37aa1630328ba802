// Adaptive-trapezoid (AI) integration of one bond over the part of the family
// node's cell inside the horizon sphere: the nested trapezoid rule of
// pdIntgManager::CalcIntg3D / CalcIntgX1-X3 / CalcTrapzdQuad
// (pdIntgManager.cpp:49-451) over the limit functions of
// pdIntgManager2.cpp:440-684.
//
// Shared by the host planner (g++ -ffp-contract=off) and the device kernels
// (nvcc -fmad=false): every operation below is one IEEE rounding in the
// order the reference's C++ evaluates it, so host and device agree bit for
// bit with the reference.  pow(x, 2.0), which g++ folds into x*x in the
// reference build, is written x*x.
//
// A bond's integral is a list of regions (pd_ai_region): the outer direction
// runs over [a, b]; the middle direction over [lim0(t), lim1(t)] for outer
// value t; the inner direction over [lim2(t, s), lim3(t, s)] for middle value
// s.  Each direction takes 2^(n-1)+1 trapezoid points (n = trapezoid index,
// 1..3); an interval of width <= 1e-10 contributes 0 and no points.
#pragma once

#include <math.h>
#include <stdint.h>

#include "../../include/pdmtel_b200.h"

#ifdef __CUDACC__
#define PD_AI_HD __host__ __device__ __forceinline__
#else
#define PD_AI_HD inline
#endif

namespace pd_ai {

// Limit codes (pd_ai_region::lim).
//  middle direction, function of the outer value t:
//    face:   2 axis + side            x_j[axis] -/+ dx/2 (side 0 low, 1 high)
//    circle: 8 + 4 (3 A + B) + 2 side + sign
//            +/- sqrt(r^2 - t^2), r^2 = delta^2 - (x_j[C] -/+ dx/2)^2, 0 where
//            negative; A the solved axis, B the outer axis, C the third one
//            (YLimitHigh/Low<A><B>Pos/Neg, pdIntgManager2.cpp:464-617)
//  inner direction, function of (t, s):
//    face:   2 axis + side
//    sphere: 8 + 2 axis + sign        +/- sqrt(delta^2 - t^2 - s^2), 0 where
//            negative (ZLimit<axis>SpherePos/Neg, pdIntgManager2.cpp:622-682)
enum { LO = 0, HI = 1, NEG = 0, POS = 1 };
constexpr uint8_t face(int axis, int side) { return (uint8_t)(2 * axis + side); }
constexpr uint8_t circle(int a, int b, int side, int sign) { return (uint8_t)(8 + 4 * (3 * a + b) + 2 * side + sign); }
constexpr uint8_t sphere(int axis, int sign) { return (uint8_t)(8 + 2 * axis + sign); }
constexpr int kMaxPerDir = 5;                       // trapezoid index 3
constexpr int kMaxRegionPoints = kMaxPerDir * kMaxPerDir * kMaxPerDir;

PD_AI_HD int points_per_dir(int n) { return n == 1 ? 2 : (n == 2 ? 3 : 5); }

// the k-th trapezoid point of [a, b] (CalcTrapzdQuad cases 1-3)
PD_AI_HD double point(int n, int k, double a, double b) {
    if (k == 0) return a;
    if (n == 1) return b;
    if (n == 2) return k == 1 ? 0.5 * (a + b) : b;
    switch (k) {
        case 1: return 0.25 * (3.0 * a + b);
        case 2: return 0.5 * (a + b);
        case 3: return 0.25 * (a + 3.0 * b);
        default: return b;
    }
}

// width factor of the rule: (b-a), 0.5 (b-a), 0.25 (b-a)
PD_AI_HD double scale(int n, double a, double b) {
    if (n == 1) return b - a;
    if (n == 2) return 0.5 * (b - a);
    return 0.25 * (b - a);
}

// running trapezoid sum: 0.5 f_0 + f_1 + ... + 0.5 f_last, left to right
PD_AI_HD void accumulate(int k, int np, const double f[3], double acc[3]) {
    if (k == 0) {
        acc[0] = 0.5 * f[0];
        acc[1] = 0.5 * f[1];
        acc[2] = 0.5 * f[2];
    } else if (k == np - 1) {
        acc[0] = acc[0] + 0.5 * f[0];
        acc[1] = acc[1] + 0.5 * f[1];
        acc[2] = acc[2] + 0.5 * f[2];
    } else {
        acc[0] = acc[0] + f[0];
        acc[1] = acc[1] + f[1];
        acc[2] = acc[2] + f[2];
    }
}

PD_AI_HD double mid_limit(int code, double t, const double xj[3], double delta, double dx) {
    if (code < 8) {
        const int ax = code >> 1;
        return (code & 1) ? xj[ax] + 0.5 * dx : xj[ax] - 0.5 * dx;
    }
    const int c = code - 8;
    const int sign = c & 1, side = (c >> 1) & 1, ab = c >> 2;
    const int A = ab / 3, B = ab % 3, C = 3 - A - B;
    const double h = side ? xj[C] + 0.5 * dx : xj[C] - 0.5 * dx;
    const double rsq = delta * delta - h * h;
    const double tt = t - 0.0;
    const double vsq = rsq - tt * tt;
    double v = vsq < 0.0 ? -1.0 : sqrt(vsq);  // SolveBinaryQuadric, pdIntgManager2.cpp:812-834
    if (v < 0.0) v = 0.0;
    return sign ? v : -v;
}

PD_AI_HD double in_limit(int code, double t, double s, const double xj[3], double delta, double dx) {
    if (code < 8) {
        const int ax = code >> 1;
        return (code & 1) ? xj[ax] + 0.5 * dx : xj[ax] - 0.5 * dx;
    }
    const double zsq = delta * delta - t * t - s * s;
    const double v = zsq < 0.0 ? 0.0 : sqrt(zsq);
    return (code & 1) ? v : -v;
}

// Integral of one region.  fn(p, k, f) evaluates the integrand at local
// point p (coordinates relative to node i) for the region's k-th evaluated
// point (pdIntgManager's _intgPointCounter, reset per region) into f[3].
// Returns the number of points evaluated.
template <class Fn>
PD_AI_HD int region(const pd_ai_region& R, int n, const double xj[3], double delta, double dx, Fn& fn, double out[3]) {
    out[0] = out[1] = out[2] = 0.0;
    if (fabs(R.a - R.b) <= 1.0e-10) return 0;
    const int np = points_per_dir(n);
    int counter = 0;
    double acc1[3] = {0.0, 0.0, 0.0};
#ifdef __CUDA_ARCH__
#pragma unroll 1
#endif
    for (int k = 0; k < np; ++k) {
        const double t = point(n, k, R.a, R.b);
        double g[3] = {0.0, 0.0, 0.0};
        const double ml = mid_limit(R.lim[0], t, xj, delta, dx);
        const double mh = mid_limit(R.lim[1], t, xj, delta, dx);
        if (!(fabs(ml - mh) <= 1.0e-10)) {
            double acc2[3] = {0.0, 0.0, 0.0};
#ifdef __CUDA_ARCH__
#pragma unroll 1
#endif
            for (int l = 0; l < np; ++l) {
                const double s = point(n, l, ml, mh);
                double h[3] = {0.0, 0.0, 0.0};
                const double zl = in_limit(R.lim[2], t, s, xj, delta, dx);
                const double zh = in_limit(R.lim[3], t, s, xj, delta, dx);
                if (!(fabs(zl - zh) <= 1.0e-10)) {
                    double acc3[3] = {0.0, 0.0, 0.0};
#ifdef __CUDA_ARCH__
#pragma unroll 1
#endif
                    for (int m = 0; m < np; ++m) {
                        double p[3], f[3];
                        p[R.axis[0]] = t;
                        p[R.axis[1]] = s;
                        p[R.axis[2]] = point(n, m, zl, zh);
                        fn(p, counter, f);
                        ++counter;
                        accumulate(m, np, f, acc3);
                    }
                    const double w = scale(n, zl, zh);
                    h[0] = w * acc3[0];
                    h[1] = w * acc3[1];
                    h[2] = w * acc3[2];
                }
                accumulate(l, np, h, acc2);
            }
            const double w = scale(n, ml, mh);
            g[0] = w * acc2[0];
            g[1] = w * acc2[1];
            g[2] = w * acc2[2];
        }
        accumulate(k, np, g, acc1);
    }
    const double w = scale(n, R.a, R.b);
    out[0] = w * acc1[0];
    out[1] = w * acc1[1];
    out[2] = w * acc1[2];
    return counter;
}

// A bond's integral: regions [r0, r1); PD_AI_ASSIGN on the first region marks
// a bond whose force is that one region's integral, else the regions are
// added to a sum that starts at 0.0 (ArrayAddition, pdIntgManager2.cpp:1811).
template <class Fn>
PD_AI_HD void bond(const pd_ai_region* regs, int64_t r0, int64_t r1, int n, const double xj[3], double delta,
                   double dx, Fn& fn, double F[3]) {
    F[0] = F[1] = F[2] = 0.0;
    if (r1 <= r0) return;
    if (regs[r0].flags & PD_AI_ASSIGN) {
        region(regs[r0], n, xj, delta, dx, fn, F);
        return;
    }
    for (int64_t r = r0; r < r1; ++r) {
        double s[3];
        region(regs[r], n, xj, delta, dx, fn, s);
        F[0] = F[0] + s[0];
        F[1] = F[1] + s[1];
        F[2] = F[2] + s[2];
    }
}

}  // namespace pd_ai
