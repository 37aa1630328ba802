// Adaptive-trapezoid (AI) integration, host side: the bond classification and
// the case analysis that split the family cell cut by the horizon sphere into
// regions (pdIntgManager::CalcConfigurationType1/2/3 and their sub-cases,
// pdIntgManager.cpp:523-3482, pdIntgManager2.cpp:836-1531), and the per-node
// MLS coefficient lists of the AI form (pdDataManager2.cpp:257-300,
// pdIntgManager2.cpp:1879-1939).
//
// The trapezoid rule is not exact, so a different split of the same volume
// integrates to different numbers: the regions, their limit functions, their
// order and the order of the three directions are the reference's, case for
// case, which is what makes the device integral equal the reference's bit for
// bit.  The regions are emitted once per bond; the device evaluates the limit
// functions (pd_ai_eval.h) on the fly.  Compiled with -ffp-contract=off.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

#include "../pd_ai_eval.h"
#include "pdDataManager.h"

namespace pdh {

namespace {

using namespace pd_ai;
enum { X = 0, Y = 1, Z = 2 };

// Geometry of one bond i -> j in the reference's family coordinates: node i
// at the origin, node j at xj (pdIntgManager.cpp:3-35).
struct Bond {
    double xj[3];
    double delta, dx;
    std::vector<pd_ai_region>* out;

    double lo(int ax) const { return xj[ax] - 0.5 * dx; }
    double hi(int ax) const { return xj[ax] + 0.5 * dx; }
    void add(int o, int m, int in, uint8_t l0, uint8_t l1, uint8_t l2, uint8_t l3, double a, double b,
             bool assign) const {
        pd_ai_region r;
        std::memset(&r, 0, sizeof(r));
        r.a = a;
        r.b = b;
        r.axis[0] = (uint8_t)o;
        r.axis[1] = (uint8_t)m;
        r.axis[2] = (uint8_t)in;
        r.lim[0] = l0;
        r.lim[1] = l1;
        r.lim[2] = l2;
        r.lim[3] = l3;
        r.flags = assign ? PD_AI_ASSIGN : 0;
        out->push_back(r);
    }
};

// sqrt(r_sq - v^2), or -1 without a real root (SolveBinaryQuadric,
// pdIntgManager2.cpp:812-834, with its centre at the origin)
double chord(double r_sq, double v) {
    const double vv = v - 0.0;
    const double s = r_sq - vv * vv;
    return s < 0.0 ? -1.0 : std::sqrt(s);
}

double unit_sign(double v) { return v == 0.0 ? 1.0 : v / std::fabs(v); }

// Intersections of the horizon sphere with the eight horizontal edges of the
// cell (FindIntersectionPointOnEightEdges, pdIntgManager2.cpp:836-973): bit
// k set when edge k is cut inside its span, with the crossing in ip[k].
// Edges: top (z high) at x low, x high (crossing in y), y low, y high
// (crossing in x), then the same four at z low.
int eight_edges(const Bond& g, double ip[8]) {
    const double xl = g.lo(X), xh = g.hi(X), yl = g.lo(Y), yh = g.hi(Y), zl = g.lo(Z), zh = g.hi(Z);
    const double n1 = unit_sign(g.xj[0]), n2 = unit_sign(g.xj[1]);
    const double d2 = g.delta * g.delta;
    int b = 0;
    const double zs[2] = {zh, zl};
    for (int face = 0; face < 2; ++face) {
        const double r_sq = d2 - zs[face] * zs[face];
        const double across[4] = {xl, xh, yl, yh};
        for (int e = 0; e < 4; ++e) {
            const int bit = 4 * face + e;
            double t = chord(r_sq, across[e]);
            if (t < 0.0) continue;
            if (e < 2) {
                t *= n2;
                if (t >= yl && t <= yh) {
                    b |= 1 << bit;
                    ip[bit] = t;
                }
            } else {
                t *= n1;
                if (t >= xl && t <= xh) {
                    b |= 1 << bit;
                    ip[bit] = t;
                }
            }
        }
    }
    return b;
}

// Intersections with the four vertical edges (FindIntersectionPointOnFourEdges,
// pdIntgManager2.cpp:975-1058): (x low, y low), (x high, y low), (x high,
// y high), (x low, y high); crossing heights in np[k].
int four_edges(const Bond& g, double np[4]) {
    const double xl = g.lo(X), xh = g.hi(X), yl = g.lo(Y), yh = g.hi(Y), zl = g.lo(Z), zh = g.hi(Z);
    const double n3 = unit_sign(g.xj[2]);
    const double d2 = g.delta * g.delta;
    const double ex[4] = {xl, xh, xh, xl}, ey[4] = {yl, yl, yh, yh};
    int b = 0;
    for (int k = 0; k < 4; ++k) {
        const double t = d2 - ex[k] * ex[k] - ey[k] * ey[k];
        if (t < 0.0) continue;
        const double z = std::sqrt(t) * n3;
        if (z >= zl && z <= zh) {
            b |= 1 << k;
            np[k] = z;
        }
    }
    return b;
}

// ---------------------------------------------------------------- type 1
// Node j on a coordinate axis (pdIntgManager.cpp:548-725 and the sub-cases
// CalcConfigurationType1Sub1-5, pdIntgManager2.cpp:1060-1399); d1 the outer
// axis (along the bond), d2 middle, d3 inner, h = dx/2.

// Sub1: the cap of the sphere inside the far half of the cell
void t1_sub1(const Bond& g, int d1, int d2, int d3, double dist) {
    const double e = dist - 0.5 * g.dx;
    const double low = -std::sqrt(g.delta * g.delta - e * e);
    const double high = std::sqrt(g.delta * g.delta - e * e);
    if (g.xj[d3] > 0.0)
        g.add(d1, d2, d3, circle(d2, d1, LO, NEG), circle(d2, d1, LO, POS), face(d3, LO), sphere(d3, POS), low,
              high, true);
    else
        g.add(d1, d2, d3, circle(d2, d1, HI, NEG), circle(d2, d1, HI, POS), sphere(d3, NEG), face(d3, HI), low,
              high, true);
}

void t1_sub2(const Bond& g, int d1, int d2, int d3, double dist) {
    const double e = dist - 0.5 * g.dx;
    const double low = -std::sqrt(g.delta * g.delta - e * e - 0.25 * g.dx * g.dx);
    const double high = std::sqrt(g.delta * g.delta - e * e - 0.25 * g.dx * g.dx);
    const double oc = g.xj[d1];
    if (g.xj[d3] > 0.0) {
        const uint8_t c0 = circle(d2, d1, LO, NEG), c1 = circle(d2, d1, LO, POS);
        g.add(d1, d2, d3, c0, c1, face(d3, LO), sphere(d3, POS), high, oc + 0.5 * g.dx, false);
        g.add(d1, d2, d3, c0, c1, face(d3, LO), sphere(d3, POS), oc - 0.5 * g.dx, low, false);
        g.add(d1, d2, d3, face(d2, LO), face(d2, HI), face(d3, LO), sphere(d3, POS), low, high, false);
    } else {
        const uint8_t c0 = circle(d2, d1, HI, NEG), c1 = circle(d2, d1, HI, POS);
        g.add(d1, d2, d3, c0, c1, sphere(d3, NEG), face(d3, HI), high, oc + 0.5 * g.dx, false);
        g.add(d1, d2, d3, c0, c1, sphere(d3, NEG), face(d3, HI), oc - 0.5 * g.dx, low, false);
        g.add(d1, d2, d3, face(d2, LO), face(d2, HI), sphere(d3, NEG), face(d3, HI), low, high, false);
    }
}

void t1_sub3(const Bond& g, int d1, int d2, int d3) {
    const double oc = g.xj[d1];
    if (g.xj[d3] > 0.0)
        g.add(d1, d2, d3, face(d2, LO), face(d2, HI), face(d3, LO), sphere(d3, POS), oc - 0.5 * g.dx,
              oc + 0.5 * g.dx, true);
    else
        g.add(d1, d2, d3, face(d2, LO), face(d2, HI), sphere(d3, NEG), face(d3, HI), oc - 0.5 * g.dx,
              oc + 0.5 * g.dx, true);
}

void t1_sub4(const Bond& g, int d1, int d2, int d3, double dist) {
    const double e = dist + 0.5 * g.dx;
    const double low = -std::sqrt(g.delta * g.delta - e * e);
    const double high = std::sqrt(g.delta * g.delta - e * e);
    const double oc = g.xj[d1];
    if (g.xj[d3] > 0.0) {
        const uint8_t zl = face(d3, LO), zs = sphere(d3, POS);
        g.add(d1, d2, d3, circle(d2, d1, HI, POS), face(d2, HI), zl, zs, low, high, false);
        g.add(d1, d2, d3, face(d2, LO), circle(d2, d1, HI, NEG), zl, zs, low, high, false);
        g.add(d1, d2, d3, face(d2, LO), face(d2, HI), zl, zs, high, oc + 0.5 * g.dx, false);
        g.add(d1, d2, d3, face(d2, LO), face(d2, HI), zl, zs, oc - 0.5 * g.dx, low, false);
        g.add(d1, d2, d3, circle(d2, d1, HI, NEG), circle(d2, d1, HI, POS), zl, zs, low, high, false);
    } else {
        const uint8_t zs = sphere(d3, NEG), zh = face(d3, HI);
        g.add(d1, d2, d3, circle(d2, d1, LO, POS), face(d2, HI), zs, zh, low, high, false);
        g.add(d1, d2, d3, face(d2, LO), circle(d2, d1, LO, NEG), zs, zh, low, high, false);
        g.add(d1, d2, d3, face(d2, LO), face(d2, HI), zs, zh, high, oc + 0.5 * g.dx, false);
        g.add(d1, d2, d3, face(d2, LO), face(d2, HI), zs, zh, oc - 0.5 * g.dx, low, false);
        g.add(d1, d2, d3, circle(d2, d1, LO, NEG), circle(d2, d1, LO, POS), zs, zh, low, high, false);
    }
}

void t1_sub5(const Bond& g, int d1, int d2, int d3, double dist) {
    const double e = dist + 0.5 * g.dx;
    const double low = -std::sqrt(g.delta * g.delta - e * e - 0.25 * g.dx * g.dx);
    const double high = std::sqrt(g.delta * g.delta - e * e - 0.25 * g.dx * g.dx);
    const double a0 = g.xj[d1] - 0.5 * g.dx, b1 = g.xj[d1] + 0.5 * g.dx;
    const uint8_t fl = face(d3, LO), fh = face(d3, HI);
    // the four corners, the centre trunk in two pieces, the core
    if (g.xj[d3] > 0.0) {
        const uint8_t zs = sphere(d3, POS);
        const uint8_t cp = circle(d2, d1, HI, POS), cn = circle(d2, d1, HI, NEG);
        g.add(d1, d2, d3, cp, face(d2, HI), fl, zs, a0, low, false);
        g.add(d1, d2, d3, cp, face(d2, HI), fl, zs, high, b1, false);
        g.add(d1, d2, d3, face(d2, LO), cn, fl, zs, a0, low, false);
        g.add(d1, d2, d3, face(d2, LO), cn, fl, zs, high, b1, false);
        g.add(d1, d2, d3, cn, cp, fl, fh, a0, low, false);
        g.add(d1, d2, d3, cn, cp, fl, fh, high, b1, false);
    } else {
        const uint8_t zs = sphere(d3, NEG);
        const uint8_t cp = circle(d2, d1, LO, POS), cn = circle(d2, d1, LO, NEG);
        g.add(d1, d2, d3, cp, face(d2, HI), zs, fh, a0, low, false);
        g.add(d1, d2, d3, cp, face(d2, HI), zs, fh, high, b1, false);
        g.add(d1, d2, d3, face(d2, LO), cn, zs, fh, a0, low, false);
        g.add(d1, d2, d3, face(d2, LO), cn, zs, fh, high, b1, false);
        g.add(d1, d2, d3, cn, cp, fl, fh, a0, low, false);
        g.add(d1, d2, d3, cn, cp, fl, fh, high, b1, false);
    }
    g.add(d1, d2, d3, face(d2, LO), face(d2, HI), fl, fh, low, high, false);
}

// CalcConfigurationType1 (pdIntgManager.cpp:548-725): the sub-case by the
// distance of node j and the edge pattern; patterns outside the listed ones
// give no force.  d1 / d2 / d3 for a node on the x, y or z axis.
void type1(const Bond& g) {
    double ip[8];
    const int b = eight_edges(g, ip);
    const double dist = std::fabs(g.xj[0] - 0.0) + std::fabs(g.xj[1] - 0.0) + std::fabs(g.xj[2] - 0.0);
    const double d = g.delta, h = 0.5 * g.dx;
    const double q1 = std::sqrt(d * d - 0.25 * g.dx * g.dx), q2 = std::sqrt(d * d - 0.5 * g.dx * g.dx);
    const double dd1 = d + h, dd2 = q1 + h, dd3 = q2 + h, dd4 = d - h, dd5 = q1 - h, dd6 = q2 - h;
    // the three axis orders a sub-case uses: x-axis node, y-axis node, z-axis node
    struct Ord { int a, b, c; };
    auto pick = [&](int code, const Ord& ox, const Ord& oy, const Ord& oz, int px, int py, int pz, int px2, int py2,
                    int pz2, Ord* o) {
        if (code == px || code == px2) { *o = ox; return true; }
        if (code == py || code == py2) { *o = oy; return true; }
        if (code == pz || code == pz2) { *o = oz; return true; }
        return false;
    };
    Ord o;
    if (dist >= dd2 && dist <= dd1) {
        if (g.xj[0] != 0.0) t1_sub1(g, Z, Y, X, dist);
        else if (g.xj[1] != 0.0) t1_sub1(g, Z, X, Y, dist);
        else t1_sub1(g, X, Y, Z, dist);
    } else if (dist >= dd3 && dist < dd2) {
        if (pick(b, {Z, Y, X}, {Z, X, Y}, {Y, X, Z}, 17, 68, 240, 34, 136, 15, &o)) t1_sub2(g, o.a, o.b, o.c, dist);
    } else if (dist >= dd4 && dist < dd3) {
        if (pick(b, {Y, Z, X}, {X, Z, Y}, {X, Y, Z}, 204, 51, 0, 204, 51, 0, &o)) t1_sub3(g, o.a, o.b, o.c);
    } else if (dist >= dd5 && dist < dd4) {
        if (pick(b, {Z, Y, X}, {Z, X, Y}, {Y, X, Z}, 204, 51, 0, 204, 51, 0, &o)) t1_sub4(g, o.a, o.b, o.c, dist);
    } else if (dist >= dd6 && dist < dd5) {
        if (pick(b, {Z, Y, X}, {Z, X, Y}, {Y, X, Z}, 238, 187, 15, 221, 119, 240, &o))
            t1_sub5(g, o.a, o.b, o.c, dist);
    }
}

// ---------------------------------------------------------------- type 2
// Node j off the axes (pdIntgManager.cpp:727-3469).

// CalcConfigurationType2Sub1 (pdIntgManager2.cpp:1413-1449): one region over
// the whole outer span, its middle and inner limits by the quadrant of
// (middle, inner) coordinates of node j
void t2_sub1(const Bond& g, int d1, int d2, int d3) {
    const double mc = g.xj[d2], ic = g.xj[d3];
    uint8_t l[4];
    if (mc > 0.0 && ic < 0.0) {
        l[0] = face(d2, LO); l[1] = circle(d2, d1, HI, POS); l[2] = sphere(d3, NEG); l[3] = face(d3, HI);
    } else if (mc > 0.0 && ic > 0.0) {
        l[0] = face(d2, LO); l[1] = circle(d2, d1, LO, POS); l[2] = face(d3, LO); l[3] = sphere(d3, POS);
    } else if (mc < 0.0 && ic > 0.0) {
        l[0] = circle(d2, d1, LO, NEG); l[1] = face(d2, HI); l[2] = face(d3, LO); l[3] = sphere(d3, POS);
    } else {
        l[0] = circle(d2, d1, HI, NEG); l[1] = face(d2, HI); l[2] = sphere(d3, NEG); l[3] = face(d3, HI);
    }
    g.add(d1, d2, d3, l[0], l[1], l[2], l[3], g.lo(d1), g.hi(d1), true);
}

// CalcConfigurationType2Sub2 (pdIntgManager2.cpp:1451-1531): two regions over
// the whole outer span
void t2_sub2(const Bond& g, int d1, int d2, int d3) {
    const double mc = g.xj[d2], ic = g.xj[d3];
    const double a = g.lo(d1), b = g.hi(d1);
    if (mc > 0.0 && ic < 0.0) {
        g.add(d1, d2, d3, circle(d2, d1, LO, POS), face(d2, HI), sphere(d3, NEG), face(d3, HI), a, b, false);
        g.add(d1, d2, d3, face(d2, LO), circle(d2, d1, LO, POS), face(d3, LO), face(d3, HI), a, b, false);
    } else if (mc > 0.0 && ic > 0.0) {
        g.add(d1, d2, d3, circle(d2, d1, HI, POS), face(d2, HI), face(d3, LO), sphere(d3, POS), a, b, false);
        g.add(d1, d2, d3, face(d2, LO), circle(d2, d1, HI, POS), face(d3, LO), face(d3, HI), a, b, false);
    } else if (mc < 0.0 && ic > 0.0) {
        g.add(d1, d2, d3, face(d2, LO), circle(d2, d1, HI, NEG), face(d3, LO), sphere(d3, POS), a, b, false);
        g.add(d1, d2, d3, circle(d2, d1, HI, NEG), face(d2, HI), face(d3, LO), face(d3, HI), a, b, false);
    } else {
        g.add(d1, d2, d3, face(d2, LO), circle(d2, d1, LO, NEG), sphere(d3, NEG), face(d3, HI), a, b, false);
        g.add(d1, d2, d3, circle(d2, d1, LO, NEG), face(d2, HI), face(d3, LO), face(d3, HI), a, b, false);
    }
}

// The case table of CalcConfigurationType2, first match wins.  A rule holds
// when the eight-edge pattern equals b; the four-edge pattern equals nb (-1:
// not consulted); cmp 1: ip[2] < ip[7], 2: ip[3] < ip[6]; the sign of node j's
// coordinate matches s (+1, -1, 0 = any) on every axis.  Its action: no force
// (ZR), regions summed (RS) or one region assigned (RD) from kT2Regs
// [first, first + count), or Type2Sub1 / Sub2 (S1, S2) with axis order
// (o, m, i).  No rule: no force.
enum Kind : uint8_t { ZR, RS, RD, S1, S2 };
struct T2Rule {
    uint8_t b;
    int8_t nb, cmp, sx, sy, sz;
    uint8_t kind, o, m, i;
    uint16_t first, count;
};
// A region of the table: axis order, the four limit codes, and the outer
// bounds: 2 axis + side (node j's cell face), 8 + k (ip[k]), 16 + k (np[k]).
struct T2Reg {
    uint8_t o, m, i, l0, l1, l2, l3, a, b;
};
constexpr uint8_t MF(int a, int s) { return face(a, s); }
constexpr uint8_t MC(int a, int b, int s, int g) { return circle(a, b, s, g); }
constexpr uint8_t IF(int a, int s) { return face(a, s); }
constexpr uint8_t IS(int a, int g) { return sphere(a, g); }
constexpr uint8_t BF(int a, int s) { return (uint8_t)(2 * a + s); }
constexpr uint8_t BI(int k) { return (uint8_t)(8 + k); }
constexpr uint8_t BN(int k) { return (uint8_t)(16 + k); }

const T2Rule kT2Rules[] = {
    { 85, -1, 0,  1,  1,  0, S1, Z, X, Y, 0, 0},
    { 85, -1, 0, -1, -1,  0, S2, Z, X, Y, 0, 0},
    {102, -1, 0, -1,  1,  0, S1, Z, X, Y, 0, 0},
    {102, -1, 0,  1, -1,  0, S2, Z, X, Y, 0, 0},
    {153, -1, 0,  1, -1,  0, S1, Z, X, Y, 0, 0},
    {153, -1, 0, -1,  1,  0, S2, Z, X, Y, 0, 0},
    {170, -1, 0, -1, -1,  0, S1, Z, X, Y, 0, 0},
    {170, -1, 0,  1,  1,  0, S2, Z, X, Y, 0, 0},
    { 12,  6, 0,  1,  0,  1, S2, Y, X, Z, 0, 0},
    { 12,  6, 0, -1,  0, -1, S1, Y, X, Z, 0, 0},
    { 12,  6, 0,  0,  0,  0, ZR, 0, 0, 0, 0, 0},
    { 12,  9, 0, -1,  0,  1, S2, Y, X, Z, 0, 0},
    { 12,  9, 0,  1,  0, -1, S1, Y, X, Z, 0, 0},
    { 12,  9, 0,  0,  0,  0, ZR, 0, 0, 0, 0, 0},
    {192,  6, 0,  1,  0, -1, S2, Y, X, Z, 0, 0},
    {192,  6, 0, -1,  0,  1, S1, Y, X, Z, 0, 0},
    {192,  6, 0,  0,  0,  0, ZR, 0, 0, 0, 0, 0},
    {192,  9, 0, -1,  0, -1, S2, Y, X, Z, 0, 0},
    {192,  9, 0,  1,  0,  1, S1, Y, X, Z, 0, 0},
    {192,  9, 0,  0,  0,  0, ZR, 0, 0, 0, 0, 0},
    {  3, 12, 0,  0,  1,  1, S2, X, Z, Y, 0, 0},
    {  3, 12, 0,  0, -1, -1, S1, X, Z, Y, 0, 0},
    {  3, 12, 0,  0,  0,  0, ZR, 0, 0, 0, 0, 0},
    {  3,  3, 0,  0, -1,  1, S2, X, Z, Y, 0, 0},
    {  3,  3, 0,  0,  1, -1, S1, X, Z, Y, 0, 0},
    {  3,  3, 0,  0,  0,  0, ZR, 0, 0, 0, 0, 0},
    { 48, 12, 0,  0,  1, -1, S2, X, Z, Y, 0, 0},
    { 48, 12, 0,  0, -1,  1, S1, X, Z, Y, 0, 0},
    { 48, 12, 0,  0,  0,  0, ZR, 0, 0, 0, 0, 0},
    { 48,  3, 0,  0, -1, -1, S2, X, Z, Y, 0, 0},
    { 48,  3, 0,  0,  1,  1, S1, X, Z, Y, 0, 0},
    { 48,  3, 0,  0,  0,  0, ZR, 0, 0, 0, 0, 0},
    {165, -1, 1,  1,  1,  1, RS, 0, 0, 0, 0, 4},
    {165, -1, 1, -1, -1, -1, RS, 0, 0, 0, 4, 4},
    {165, -1, 1,  0,  0,  0, ZR, 0, 0, 0, 0, 0},
    {165, -1, 0,  1,  1,  1, RS, 0, 0, 0, 8, 4},
    {165, -1, 0, -1, -1, -1, RS, 0, 0, 0, 12, 4},
    { 90, -1, 2,  1,  1, -1, RS, 0, 0, 0, 16, 4},
    { 90, -1, 2, -1, -1,  1, RS, 0, 0, 0, 20, 4},
    { 90, -1, 2,  0,  0,  0, ZR, 0, 0, 0, 0, 0},
    { 90, -1, 0,  1,  1, -1, RS, 0, 0, 0, 24, 4},
    { 90, -1, 0, -1, -1,  1, RS, 0, 0, 0, 28, 4},
    {150, -1, 1, -1,  1,  1, RS, 0, 0, 0, 32, 4},
    {150, -1, 1,  1, -1, -1, RS, 0, 0, 0, 36, 4},
    {150, -1, 1,  0,  0,  0, ZR, 0, 0, 0, 0, 0},
    {150, -1, 0, -1,  1,  1, RS, 0, 0, 0, 40, 4},
    {150, -1, 0,  1, -1, -1, RS, 0, 0, 0, 44, 4},
    {105, -1, 2, -1,  1, -1, RS, 0, 0, 0, 48, 4},
    {105, -1, 2,  1, -1,  1, RS, 0, 0, 0, 52, 4},
    {105, -1, 2,  0,  0,  0, ZR, 0, 0, 0, 0, 0},
    {105, -1, 0, -1,  1, -1, RS, 0, 0, 0, 56, 4},
    {105, -1, 0,  1, -1,  1, RS, 0, 0, 0, 60, 4},
    { 10,  4, 0,  1,  1,  1, RS, 0, 0, 0, 64, 3},
    { 10,  4, 0, -1, -1, -1, RD, 0, 0, 0, 67, 1},
    { 10,  4, 0,  0,  0,  0, ZR, 0, 0, 0, 0, 0},
    { 10, 11, 0,  1,  1, -1, RS, 0, 0, 0, 68, 2},
    { 10, 11, 0, -1, -1,  1, RS, 0, 0, 0, 70, 3},
    { 10, 11, 0,  0,  0,  0, ZR, 0, 0, 0, 0, 0},
    {160,  4, 0,  1,  1, -1, RS, 0, 0, 0, 73, 3},
    {160,  4, 0, -1, -1,  1, RD, 0, 0, 0, 76, 1},
    {160,  4, 0,  0,  0,  0, ZR, 0, 0, 0, 0, 0},
    {160, 11, 0,  1,  1,  1, RS, 0, 0, 0, 77, 2},
    {160, 11, 0, -1, -1, -1, RS, 0, 0, 0, 79, 3},
    {160, 11, 0,  0,  0,  0, ZR, 0, 0, 0, 0, 0},
    {  9,  8, 0, -1,  1,  1, RS, 0, 0, 0, 82, 3},
    {  9,  8, 0,  1, -1, -1, RD, 0, 0, 0, 85, 1},
    {  9,  8, 0,  0,  0,  0, ZR, 0, 0, 0, 0, 0},
    {  9,  7, 0, -1,  1, -1, RS, 0, 0, 0, 86, 2},
    {  9,  7, 0,  1, -1,  1, RS, 0, 0, 0, 88, 3},
    {  9,  7, 0,  0,  0,  0, ZR, 0, 0, 0, 0, 0},
    {144,  8, 0, -1,  1, -1, RS, 0, 0, 0, 91, 3},
    {144,  8, 0,  1, -1,  1, RD, 0, 0, 0, 94, 1},
    {144,  8, 0,  0,  0,  0, ZR, 0, 0, 0, 0, 0},
    {144,  7, 0, -1,  1,  1, RS, 0, 0, 0, 95, 2},
    {144,  7, 0,  1, -1, -1, RS, 0, 0, 0, 97, 3},
    {144,  7, 0,  0,  0,  0, ZR, 0, 0, 0, 0, 0},
    {  6,  2, 0,  1, -1,  1, RS, 0, 0, 0, 100, 3},
    {  6,  2, 0, -1,  1, -1, RD, 0, 0, 0, 103, 1},
    {  6,  2, 0,  0,  0,  0, ZR, 0, 0, 0, 0, 0},
    {  6, 13, 0,  1, -1, -1, RS, 0, 0, 0, 104, 2},
    {  6, 13, 0, -1,  1,  1, RS, 0, 0, 0, 106, 3},
    {  6, 13, 0,  0,  0,  0, ZR, 0, 0, 0, 0, 0},
    {  5,  1, 0, -1, -1,  1, RS, 0, 0, 0, 109, 3},
    {  5,  1, 0,  1,  1, -1, RD, 0, 0, 0, 112, 1},
    {  5,  1, 0,  0,  0,  0, ZR, 0, 0, 0, 0, 0},
    {  5, 14, 0, -1, -1, -1, RS, 0, 0, 0, 113, 2},
    {  5, 14, 0,  1,  1,  1, RS, 0, 0, 0, 115, 3},
    {  5, 14, 0,  0,  0,  0, ZR, 0, 0, 0, 0, 0},
    { 96,  2, 0,  1, -1, -1, RS, 0, 0, 0, 118, 3},
    { 96,  2, 0, -1,  1,  1, RD, 0, 0, 0, 121, 1},
    { 96,  2, 0,  0,  0,  0, ZR, 0, 0, 0, 0, 0},
    { 96, 13, 0,  1, -1,  1, RS, 0, 0, 0, 122, 2},
    { 96, 13, 0, -1,  1, -1, RS, 0, 0, 0, 124, 3},
    { 96, 13, 0,  0,  0,  0, ZR, 0, 0, 0, 0, 0},
    { 80,  1, 0, -1, -1, -1, RS, 0, 0, 0, 127, 3},
    { 80,  1, 0,  1,  1,  1, RD, 0, 0, 0, 130, 1},
    { 80,  1, 0,  0,  0,  0, ZR, 0, 0, 0, 0, 0},
    { 80, 14, 0, -1, -1,  1, RS, 0, 0, 0, 131, 2},
    { 80, 14, 0,  1,  1, -1, RS, 0, 0, 0, 133, 3},
    { 80, 14, 0,  0,  0,  0, ZR, 0, 0, 0, 0, 0},
    { 53, -1, 0,  1,  1,  1, RS, 0, 0, 0, 136, 2},
    { 53, -1, 0, -1, -1, -1, RS, 0, 0, 0, 138, 3},
    { 83, -1, 0,  1,  1, -1, RS, 0, 0, 0, 141, 2},
    { 83, -1, 0, -1, -1,  1, RS, 0, 0, 0, 143, 3},
    { 54, -1, 0, -1,  1,  1, RS, 0, 0, 0, 146, 2},
    { 54, -1, 0,  1, -1, -1, RS, 0, 0, 0, 148, 3},
    { 99, -1, 0, -1,  1, -1, RS, 0, 0, 0, 151, 2},
    { 99, -1, 0,  1, -1,  1, RS, 0, 0, 0, 153, 3},
    { 57, -1, 0,  1, -1,  1, RS, 0, 0, 0, 156, 2},
    { 57, -1, 0, -1,  1, -1, RS, 0, 0, 0, 158, 3},
    {147, -1, 0,  1, -1, -1, RS, 0, 0, 0, 161, 2},
    {147, -1, 0, -1,  1,  1, RS, 0, 0, 0, 163, 3},
    { 58, -1, 0, -1, -1,  1, RS, 0, 0, 0, 166, 2},
    { 58, -1, 0,  1,  1, -1, RS, 0, 0, 0, 168, 3},
    {163, -1, 0, -1, -1, -1, RS, 0, 0, 0, 171, 2},
    {163, -1, 0,  1,  1,  1, RS, 0, 0, 0, 173, 3},
    {204, -1, 0,  1,  0,  0, RD, 0, 0, 0, 176, 1},
    {204, -1, 0,  0,  0,  0, RD, 0, 0, 0, 177, 1},
    { 51, -1, 0,  0,  1,  0, RD, 0, 0, 0, 178, 1},
    { 51, -1, 0,  0,  0,  0, RD, 0, 0, 0, 179, 1},
    {  0, 15, 0,  0,  0,  1, RD, 0, 0, 0, 180, 1},
    {  0, 15, 0,  0,  0,  0, RD, 0, 0, 0, 181, 1},
    {197,  8, 0,  1,  1,  1, RS, 0, 0, 0, 182, 2},
    {197, -1, 0,  1,  1,  1, ZR, 0, 0, 0, 0, 0},
    {197,  8, 0, -1, -1, -1, RS, 0, 0, 0, 184, 3},
    {197, -1, 0, -1, -1, -1, ZR, 0, 0, 0, 0, 0},
    { 92,  8, 0,  1,  1, -1, RS, 0, 0, 0, 187, 2},
    { 92, -1, 0,  1,  1, -1, ZR, 0, 0, 0, 0, 0},
    { 92,  8, 0, -1, -1,  1, RS, 0, 0, 0, 189, 3},
    { 92, -1, 0, -1, -1,  1, ZR, 0, 0, 0, 0, 0},
    {201,  1, 0,  1, -1,  1, RS, 0, 0, 0, 192, 2},
    {201, -1, 0,  1, -1,  1, ZR, 0, 0, 0, 0, 0},
    {201,  1, 0, -1,  1, -1, RS, 0, 0, 0, 194, 3},
    {201, -1, 0, -1,  1, -1, ZR, 0, 0, 0, 0, 0},
    {156,  1, 0,  1, -1, -1, RS, 0, 0, 0, 197, 2},
    {156, -1, 0,  1, -1, -1, ZR, 0, 0, 0, 0, 0},
    {156,  1, 0, -1,  1,  1, RS, 0, 0, 0, 199, 3},
    {156, -1, 0, -1,  1,  1, ZR, 0, 0, 0, 0, 0},
    {198,  4, 0, -1,  1,  1, RS, 0, 0, 0, 202, 2},
    {198, -1, 0, -1,  1,  1, ZR, 0, 0, 0, 0, 0},
    {198,  4, 0,  1, -1, -1, RS, 0, 0, 0, 204, 3},
    {198, -1, 0,  1, -1, -1, ZR, 0, 0, 0, 0, 0},
    {108,  4, 0, -1,  1, -1, RS, 0, 0, 0, 207, 2},
    {108, -1, 0, -1,  1, -1, ZR, 0, 0, 0, 0, 0},
    {108,  4, 0,  1, -1,  1, RS, 0, 0, 0, 209, 3},
    {108, -1, 0,  1, -1,  1, ZR, 0, 0, 0, 0, 0},
    {202,  2, 0, -1, -1,  1, RS, 0, 0, 0, 212, 2},
    {202, -1, 0, -1, -1,  1, ZR, 0, 0, 0, 0, 0},
    {202,  2, 0,  1,  1, -1, RS, 0, 0, 0, 214, 3},
    {202, -1, 0,  1,  1, -1, ZR, 0, 0, 0, 0, 0},
    {172,  2, 0, -1, -1, -1, RS, 0, 0, 0, 217, 2},
    {172, -1, 0, -1, -1, -1, ZR, 0, 0, 0, 0, 0},
    {172,  2, 0,  1,  1,  1, RS, 0, 0, 0, 219, 3},
    {172, -1, 0,  1,  1,  1, ZR, 0, 0, 0, 0, 0},
};

const T2Reg kT2Regs[] = {
    {X, Y, Z, MC(Y,X,HI,POS), MF(Y,HI), IF(Z,LO), IS(Z,POS), BF(X,LO), BI(2)},
    {X, Y, Z, MF(Y,LO), MF(Y,HI), IF(Z,LO), IS(Z,POS), BI(2), BI(7)},
    {X, Y, Z, MF(Y,LO), MC(Y,X,LO,POS), IF(Z,LO), IS(Z,POS), BI(7), BF(X,HI)},
    {X, Y, Z, MF(Y,LO), MC(Y,X,HI,POS), IF(Z,LO), IF(Z,HI), BF(X,LO), BI(2)},
    {X, Y, Z, MC(Y,X,HI,NEG), MF(Y,HI), IS(Z,NEG), IF(Z,HI), BF(X,LO), BI(2)},
    {X, Y, Z, MF(Y,LO), MF(Y,HI), IS(Z,NEG), IF(Z,HI), BI(2), BI(7)},
    {X, Y, Z, MF(Y,LO), MC(Y,X,LO,NEG), IS(Z,NEG), IF(Z,HI), BI(7), BF(X,HI)},
    {X, Y, Z, MC(Y,X,LO,NEG), MF(Y,HI), IF(Z,LO), IF(Z,HI), BI(7), BF(X,HI)},
    {X, Y, Z, MC(Y,X,HI,POS), MF(Y,HI), IF(Z,LO), IS(Z,POS), BF(X,LO), BI(7)},
    {X, Y, Z, MC(Y,X,HI,POS), MC(Y,X,LO,POS), IF(Z,LO), IS(Z,POS), BI(7), BI(2)},
    {X, Y, Z, MF(Y,LO), MC(Y,X,LO,POS), IF(Z,LO), IS(Z,POS), BI(2), BF(X,HI)},
    {X, Y, Z, MF(Y,LO), MC(Y,X,HI,POS), IF(Z,LO), IF(Z,HI), BF(X,LO), BI(2)},
    {X, Y, Z, MC(Y,X,HI,NEG), MF(Y,HI), IS(Z,NEG), IF(Z,HI), BF(X,LO), BI(7)},
    {X, Y, Z, MC(Y,X,HI,NEG), MC(Y,X,LO,NEG), IS(Z,NEG), IF(Z,HI), BI(7), BI(2)},
    {X, Y, Z, MF(Y,LO), MC(Y,X,LO,NEG), IS(Z,NEG), IF(Z,HI), BI(2), BF(X,HI)},
    {X, Y, Z, MC(Y,X,LO,NEG), MF(Y,HI), IF(Z,LO), IF(Z,HI), BI(7), BF(X,HI)},
    {X, Z, Y, MF(Z,LO), MC(Z,X,HI,NEG), IF(Y,LO), IS(Y,POS), BF(X,LO), BI(3)},
    {X, Z, Y, MF(Z,LO), MF(Z,HI), IF(Y,LO), IS(Y,POS), BI(3), BI(6)},
    {X, Z, Y, MC(Z,X,LO,NEG), MF(Z,HI), IF(Y,LO), IS(Y,POS), BI(6), BF(X,HI)},
    {X, Z, Y, MC(Z,X,HI,NEG), MF(Z,HI), IF(Y,LO), IF(Y,HI), BF(X,LO), BI(3)},
    {X, Z, Y, MF(Z,LO), MC(Z,X,HI,POS), IS(Y,NEG), IF(Y,HI), BF(X,LO), BI(3)},
    {X, Z, Y, MF(Z,LO), MF(Z,HI), IS(Y,NEG), IF(Y,HI), BI(3), BI(6)},
    {X, Z, Y, MC(Z,X,LO,POS), MF(Z,HI), IS(Y,NEG), IF(Y,HI), BI(6), BF(X,HI)},
    {X, Z, Y, MF(Z,LO), MC(Z,X,LO,POS), IF(Y,LO), IF(Y,HI), BI(6), BF(X,HI)},
    {X, Z, Y, MF(Z,LO), MC(Z,X,HI,NEG), IF(Y,LO), IS(Y,POS), BF(X,LO), BI(6)},
    {X, Z, Y, MC(Z,X,LO,NEG), MC(Z,X,HI,NEG), IF(Y,LO), IS(Y,POS), BI(6), BI(3)},
    {X, Z, Y, MC(Z,X,LO,NEG), MF(Z,HI), IF(Y,LO), IS(Y,POS), BI(3), BF(X,HI)},
    {X, Z, Y, MC(Z,X,HI,NEG), MF(Z,HI), IF(Y,LO), IF(Y,HI), BF(X,LO), BI(3)},
    {X, Z, Y, MF(Z,LO), MC(Z,X,HI,POS), IS(Y,NEG), IF(Y,HI), BF(X,LO), BI(6)},
    {X, Z, Y, MC(Z,X,LO,POS), MC(Z,X,HI,POS), IS(Y,NEG), IF(Y,HI), BI(6), BI(3)},
    {X, Z, Y, MC(Z,X,LO,POS), MF(Z,HI), IS(Y,NEG), IF(Y,HI), BI(3), BF(X,HI)},
    {X, Z, Y, MF(Z,LO), MC(Z,X,LO,POS), IF(Y,LO), IF(Y,HI), BI(6), BF(X,HI)},
    {X, Z, Y, MC(Z,X,HI,POS), MF(Z,HI), IF(Y,LO), IS(Y,POS), BI(7), BF(X,HI)},
    {X, Z, Y, MF(Z,LO), MF(Z,HI), IF(Y,LO), IS(Y,POS), BI(2), BI(7)},
    {X, Z, Y, MF(Z,LO), MC(Z,X,LO,POS), IF(Y,LO), IS(Y,POS), BF(X,LO), BI(2)},
    {X, Z, Y, MF(Z,LO), MC(Z,X,HI,POS), IF(Y,LO), IF(Y,HI), BI(7), BF(X,HI)},
    {X, Z, Y, MC(Z,X,HI,NEG), MF(Z,HI), IS(Y,NEG), IF(Y,HI), BI(7), BF(X,HI)},
    {X, Z, Y, MF(Z,LO), MF(Z,HI), IS(Y,NEG), IF(Y,HI), BI(2), BI(7)},
    {X, Z, Y, MF(Z,LO), MC(Z,X,LO,NEG), IS(Y,NEG), IF(Y,HI), BF(X,LO), BI(2)},
    {X, Z, Y, MC(Z,X,LO,NEG), MF(Z,HI), IF(Y,LO), IF(Y,HI), BF(X,LO), BI(2)},
    {X, Z, Y, MC(Z,X,HI,POS), MF(Z,HI), IF(Y,LO), IS(Y,POS), BI(2), BF(X,HI)},
    {X, Z, Y, MC(Z,X,HI,POS), MC(Z,X,LO,POS), IF(Y,LO), IS(Y,POS), BI(7), BI(2)},
    {X, Z, Y, MF(Z,LO), MC(Z,X,LO,POS), IF(Y,LO), IS(Y,POS), BF(X,LO), BI(7)},
    {X, Z, Y, MF(Z,LO), MC(Z,X,HI,POS), IF(Y,LO), IF(Y,HI), BI(7), BF(X,HI)},
    {X, Z, Y, MC(Z,X,HI,NEG), MF(Z,HI), IS(Y,NEG), IF(Y,HI), BI(2), BF(X,HI)},
    {X, Z, Y, MC(Z,X,HI,NEG), MC(Z,X,LO,NEG), IS(Y,NEG), IF(Y,HI), BI(7), BI(2)},
    {X, Z, Y, MF(Z,LO), MC(Z,X,LO,NEG), IS(Y,NEG), IF(Y,HI), BF(X,LO), BI(7)},
    {X, Z, Y, MC(Z,X,LO,NEG), MF(Z,HI), IF(Y,LO), IF(Y,HI), BF(X,LO), BI(2)},
    {X, Y, Z, MF(Y,LO), MC(Y,X,HI,POS), IS(Z,NEG), IF(Z,HI), BF(X,LO), BI(3)},
    {X, Y, Z, MF(Y,LO), MF(Y,HI), IS(Z,NEG), IF(Z,HI), BI(3), BI(6)},
    {X, Y, Z, MC(Y,X,LO,POS), MF(Y,HI), IS(Z,NEG), IF(Z,HI), BI(6), BF(X,HI)},
    {X, Y, Z, MF(Y,LO), MC(Y,X,LO,POS), IF(Z,LO), IF(Z,HI), BI(6), BF(X,HI)},
    {X, Y, Z, MF(Y,LO), MC(Y,X,HI,NEG), IF(Z,LO), IS(Z,POS), BF(X,LO), BI(3)},
    {X, Y, Z, MF(Y,LO), MF(Y,HI), IF(Z,LO), IS(Z,POS), BI(3), BI(6)},
    {X, Y, Z, MC(Y,X,LO,NEG), MF(Y,HI), IF(Z,LO), IS(Z,POS), BI(6), BF(X,HI)},
    {X, Y, Z, MC(Y,X,HI,NEG), MF(Y,HI), IF(Z,LO), IF(Z,HI), BF(X,LO), BI(3)},
    {X, Y, Z, MF(Y,LO), MC(Y,X,HI,POS), IS(Z,NEG), IF(Z,HI), BF(X,LO), BI(6)},
    {X, Y, Z, MC(Y,X,LO,POS), MC(Y,X,HI,POS), IS(Z,NEG), IF(Z,HI), BI(6), BI(3)},
    {X, Y, Z, MC(Y,X,LO,POS), MF(Y,HI), IS(Z,NEG), IF(Z,HI), BI(3), BF(X,HI)},
    {X, Y, Z, MF(Y,LO), MC(Y,X,LO,POS), IF(Z,LO), IF(Z,HI), BI(6), BF(X,HI)},
    {X, Y, Z, MF(Y,LO), MC(Y,X,HI,NEG), IF(Z,LO), IS(Z,POS), BF(X,LO), BI(6)},
    {X, Y, Z, MC(Y,X,LO,NEG), MC(Y,X,HI,NEG), IF(Z,LO), IS(Z,POS), BI(6), BI(3)},
    {X, Y, Z, MC(Y,X,LO,NEG), MF(Y,HI), IF(Z,LO), IS(Z,POS), BI(3), BF(X,HI)},
    {X, Y, Z, MC(Y,X,HI,NEG), MF(Y,HI), IF(Z,LO), IF(Z,HI), BF(X,LO), BI(3)},
    {X, Z, Y, MC(Z,X,HI,POS), MF(Z,HI), IF(Y,LO), IS(Y,POS), BI(3), BF(X,HI)},
    {X, Z, Y, MF(Z,LO), MC(Z,X,HI,POS), IF(Y,LO), IF(Y,HI), BI(3), BF(X,HI)},
    {X, Z, Y, MF(Z,LO), MF(Z,HI), IF(Y,LO), IF(Y,HI), BF(X,LO), BI(3)},
    {X, Z, Y, MC(Z,X,HI,NEG), MF(Z,HI), IS(Y,NEG), IF(Y,HI), BI(3), BF(X,HI)},
    {X, Y, Z, MF(Y,LO), MC(Y,X,HI,POS), IS(Z,NEG), IF(Z,HI), BI(3), BF(X,HI)},
    {X, Y, Z, MF(Y,LO), MF(Y,HI), IS(Z,NEG), IF(Z,HI), BF(X,LO), BI(3)},
    {X, Y, Z, MF(Y,LO), MC(Y,X,HI,NEG), IF(Z,LO), IS(Z,POS), BI(3), BF(X,HI)},
    {X, Y, Z, MF(Y,LO), MF(Y,HI), IF(Z,LO), IS(Z,POS), BF(X,LO), BI(3)},
    {X, Y, Z, MC(Y,X,HI,NEG), MF(Y,HI), IF(Z,LO), IF(Z,HI), BI(3), BF(X,HI)},
    {X, Z, Y, MF(Z,LO), MC(Z,X,HI,NEG), IF(Y,LO), IS(Y,POS), BI(7), BF(X,HI)},
    {X, Z, Y, MC(Z,X,HI,NEG), MF(Z,HI), IF(Y,LO), IF(Y,HI), BI(7), BF(X,HI)},
    {X, Z, Y, MF(Z,LO), MF(Z,HI), IF(Y,LO), IF(Y,HI), BF(X,LO), BI(7)},
    {X, Z, Y, MF(Z,LO), MC(Z,X,HI,POS), IS(Y,NEG), IF(Y,HI), BI(7), BF(X,HI)},
    {X, Y, Z, MF(Y,LO), MC(Y,X,LO,POS), IF(Z,LO), IS(Z,POS), BI(7), BF(X,HI)},
    {X, Y, Z, MF(Y,LO), MF(Y,HI), IF(Z,LO), IS(Z,POS), BF(X,LO), BI(7)},
    {X, Y, Z, MF(Y,LO), MC(Y,X,LO,NEG), IS(Z,NEG), IF(Z,HI), BI(7), BF(X,HI)},
    {X, Y, Z, MF(Y,LO), MF(Y,HI), IS(Z,NEG), IF(Z,HI), BF(X,LO), BI(7)},
    {X, Y, Z, MC(Y,X,LO,NEG), MF(Y,HI), IF(Z,LO), IF(Z,HI), BI(7), BF(X,HI)},
    {X, Z, Y, MC(Z,X,HI,POS), MF(Z,HI), IF(Y,LO), IS(Y,POS), BF(X,LO), BI(3)},
    {X, Z, Y, MF(Z,LO), MC(Z,X,HI,POS), IF(Y,LO), IF(Y,HI), BF(X,LO), BI(3)},
    {X, Z, Y, MF(Z,LO), MF(Z,HI), IF(Y,LO), IF(Y,HI), BI(3), BF(X,HI)},
    {X, Z, Y, MC(Z,X,HI,NEG), MF(Z,HI), IS(Y,NEG), IF(Y,HI), BF(X,LO), BI(3)},
    {X, Y, Z, MF(Y,LO), MC(Y,X,HI,POS), IS(Z,NEG), IF(Z,HI), BF(X,LO), BI(3)},
    {X, Y, Z, MF(Y,LO), MF(Y,HI), IS(Z,NEG), IF(Z,HI), BI(3), BF(X,HI)},
    {X, Y, Z, MF(Y,LO), MC(Y,X,HI,NEG), IF(Z,LO), IS(Z,POS), BF(X,LO), BI(3)},
    {X, Y, Z, MF(Y,LO), MF(Y,HI), IF(Z,LO), IS(Z,POS), BI(3), BF(X,HI)},
    {X, Y, Z, MC(Y,X,HI,NEG), MF(Y,HI), IF(Z,LO), IF(Z,HI), BF(X,LO), BI(3)},
    {X, Z, Y, MF(Z,LO), MC(Z,X,HI,NEG), IF(Y,LO), IS(Y,POS), BF(X,LO), BI(7)},
    {X, Z, Y, MC(Z,X,HI,NEG), MF(Z,HI), IF(Y,LO), IF(Y,HI), BF(X,LO), BI(7)},
    {X, Z, Y, MF(Z,LO), MF(Z,HI), IF(Y,LO), IF(Y,HI), BI(7), BF(X,HI)},
    {X, Z, Y, MF(Z,LO), MC(Z,X,HI,POS), IS(Y,NEG), IF(Y,HI), BF(X,LO), BI(7)},
    {X, Y, Z, MF(Y,LO), MC(Y,X,LO,POS), IF(Z,LO), IS(Z,POS), BF(X,LO), BI(7)},
    {X, Y, Z, MF(Y,LO), MF(Y,HI), IF(Z,LO), IS(Z,POS), BI(7), BF(X,HI)},
    {X, Y, Z, MF(Y,LO), MC(Y,X,LO,NEG), IS(Z,NEG), IF(Z,HI), BF(X,LO), BI(7)},
    {X, Y, Z, MF(Y,LO), MF(Y,HI), IS(Z,NEG), IF(Z,HI), BI(7), BF(X,HI)},
    {X, Y, Z, MC(Y,X,LO,NEG), MF(Y,HI), IF(Z,LO), IF(Z,HI), BF(X,LO), BI(7)},
    {X, Z, Y, MC(Z,X,LO,POS), MF(Z,HI), IS(Y,NEG), IF(Y,HI), BI(2), BF(X,HI)},
    {X, Z, Y, MF(Z,LO), MC(Z,X,LO,POS), IF(Y,LO), IF(Y,HI), BI(2), BF(X,HI)},
    {X, Z, Y, MF(Z,LO), MF(Z,HI), IF(Y,LO), IF(Y,HI), BF(X,LO), BI(2)},
    {X, Z, Y, MC(Z,X,LO,NEG), MF(Z,HI), IF(Y,LO), IS(Y,POS), BI(2), BF(X,HI)},
    {X, Y, Z, MC(Y,X,HI,NEG), MF(Y,HI), IS(Z,NEG), IF(Z,HI), BI(2), BF(X,HI)},
    {X, Y, Z, MF(Y,LO), MF(Y,HI), IS(Z,NEG), IF(Z,HI), BF(X,LO), BI(2)},
    {X, Y, Z, MC(Y,X,HI,POS), MF(Y,HI), IF(Z,LO), IS(Z,POS), BI(2), BF(X,HI)},
    {X, Y, Z, MF(Y,LO), MF(Y,HI), IF(Z,LO), IS(Z,POS), BF(X,LO), BI(2)},
    {X, Y, Z, MF(Y,LO), MC(Y,X,HI,POS), IF(Z,LO), IF(Z,HI), BI(2), BF(X,HI)},
    {X, Z, Y, MC(Z,X,LO,POS), MF(Z,HI), IS(Y,NEG), IF(Y,HI), BF(X,LO), BI(2)},
    {X, Z, Y, MF(Z,LO), MC(Z,X,LO,POS), IF(Y,LO), IF(Y,HI), BF(X,LO), BI(2)},
    {X, Z, Y, MF(Z,LO), MF(Z,HI), IF(Y,LO), IF(Y,HI), BI(2), BF(X,HI)},
    {X, Z, Y, MC(Z,X,LO,NEG), MF(Z,HI), IF(Y,LO), IS(Y,POS), BF(X,LO), BI(2)},
    {X, Y, Z, MC(Y,X,HI,NEG), MF(Y,HI), IS(Z,NEG), IF(Z,HI), BF(X,LO), BI(2)},
    {X, Y, Z, MF(Y,LO), MF(Y,HI), IS(Z,NEG), IF(Z,HI), BI(2), BF(X,HI)},
    {X, Y, Z, MC(Y,X,HI,POS), MF(Y,HI), IF(Z,LO), IS(Z,POS), BF(X,LO), BI(2)},
    {X, Y, Z, MF(Y,LO), MF(Y,HI), IF(Z,LO), IS(Z,POS), BI(2), BF(X,HI)},
    {X, Y, Z, MF(Y,LO), MC(Y,X,HI,POS), IF(Z,LO), IF(Z,HI), BF(X,LO), BI(2)},
    {X, Z, Y, MF(Z,LO), MC(Z,X,LO,NEG), IS(Y,NEG), IF(Y,HI), BI(6), BF(X,HI)},
    {X, Z, Y, MC(Z,X,LO,NEG), MF(Z,HI), IF(Y,LO), IF(Y,HI), BI(6), BF(X,HI)},
    {X, Z, Y, MF(Z,LO), MF(Z,HI), IF(Y,LO), IF(Y,HI), BF(X,LO), BI(6)},
    {X, Z, Y, MF(Z,LO), MC(Z,X,LO,POS), IF(Y,LO), IS(Y,POS), BI(6), BF(X,HI)},
    {X, Y, Z, MC(Y,X,LO,NEG), MF(Y,HI), IF(Z,LO), IS(Z,POS), BI(6), BF(X,HI)},
    {X, Y, Z, MF(Y,LO), MF(Y,HI), IF(Z,LO), IS(Z,POS), BF(X,LO), BI(6)},
    {X, Y, Z, MC(Y,X,LO,POS), MF(Y,HI), IS(Z,NEG), IF(Z,HI), BI(6), BF(X,HI)},
    {X, Y, Z, MF(Y,LO), MF(Y,HI), IS(Z,NEG), IF(Z,HI), BF(X,LO), BI(6)},
    {X, Y, Z, MF(Y,LO), MC(Y,X,LO,POS), IF(Z,LO), IF(Z,HI), BI(6), BF(X,HI)},
    {X, Z, Y, MF(Z,LO), MC(Z,X,LO,NEG), IS(Y,NEG), IF(Y,HI), BF(X,LO), BI(6)},
    {X, Z, Y, MC(Z,X,LO,NEG), MF(Z,HI), IF(Y,LO), IF(Y,HI), BF(X,LO), BI(6)},
    {X, Z, Y, MF(Z,LO), MF(Z,HI), IF(Y,LO), IF(Y,HI), BI(6), BF(X,HI)},
    {X, Z, Y, MF(Z,LO), MC(Z,X,LO,POS), IF(Y,LO), IS(Y,POS), BF(X,LO), BI(6)},
    {X, Y, Z, MC(Y,X,LO,NEG), MF(Y,HI), IF(Z,LO), IS(Z,POS), BF(X,LO), BI(6)},
    {X, Y, Z, MF(Y,LO), MF(Y,HI), IF(Z,LO), IS(Z,POS), BI(6), BF(X,HI)},
    {X, Y, Z, MC(Y,X,LO,POS), MF(Y,HI), IS(Z,NEG), IF(Z,HI), BF(X,LO), BI(6)},
    {X, Y, Z, MF(Y,LO), MF(Y,HI), IS(Z,NEG), IF(Z,HI), BI(6), BF(X,HI)},
    {X, Y, Z, MF(Y,LO), MC(Y,X,LO,POS), IF(Z,LO), IF(Z,HI), BF(X,LO), BI(6)},
    {X, Z, Y, MF(Z,LO), MC(Z,X,LO,POS), IF(Y,LO), IS(Y,POS), BI(2), BF(X,HI)},
    {X, Z, Y, MF(Z,LO), MF(Z,HI), IF(Y,LO), IS(Y,POS), BF(X,LO), BI(2)},
    {X, Z, Y, MF(Z,LO), MC(Z,X,LO,NEG), IS(Y,NEG), IF(Y,HI), BI(2), BF(X,HI)},
    {X, Z, Y, MF(Z,LO), MF(Z,HI), IS(Y,NEG), IF(Y,HI), BF(X,LO), BI(2)},
    {X, Z, Y, MC(Z,X,LO,NEG), MF(Z,HI), IF(Y,LO), IF(Y,HI), BI(2), BF(X,HI)},
    {X, Z, Y, MC(Z,X,LO,NEG), MF(Z,HI), IF(Y,LO), IS(Y,POS), BI(6), BF(X,HI)},
    {X, Z, Y, MF(Z,LO), MF(Z,HI), IF(Y,LO), IS(Y,POS), BF(X,LO), BI(6)},
    {X, Z, Y, MC(Z,X,LO,POS), MF(Z,HI), IS(Y,NEG), IF(Y,HI), BI(6), BF(X,HI)},
    {X, Z, Y, MF(Z,LO), MF(Z,HI), IS(Y,NEG), IF(Y,HI), BF(X,LO), BI(6)},
    {X, Z, Y, MF(Z,LO), MC(Z,X,LO,POS), IF(Y,LO), IF(Y,HI), BI(6), BF(X,HI)},
    {X, Z, Y, MF(Z,LO), MC(Z,X,LO,POS), IF(Y,LO), IS(Y,POS), BF(X,LO), BI(2)},
    {X, Z, Y, MF(Z,LO), MF(Z,HI), IF(Y,LO), IS(Y,POS), BI(2), BF(X,HI)},
    {X, Z, Y, MF(Z,LO), MC(Z,X,LO,NEG), IS(Y,NEG), IF(Y,HI), BF(X,LO), BI(2)},
    {X, Z, Y, MF(Z,LO), MF(Z,HI), IS(Y,NEG), IF(Y,HI), BI(2), BF(X,HI)},
    {X, Z, Y, MC(Z,X,LO,NEG), MF(Z,HI), IF(Y,LO), IF(Y,HI), BF(X,LO), BI(2)},
    {X, Z, Y, MC(Z,X,LO,NEG), MF(Z,HI), IF(Y,LO), IS(Y,POS), BF(X,LO), BI(6)},
    {X, Z, Y, MF(Z,LO), MF(Z,HI), IF(Y,LO), IS(Y,POS), BI(6), BF(X,HI)},
    {X, Z, Y, MC(Z,X,LO,POS), MF(Z,HI), IS(Y,NEG), IF(Y,HI), BF(X,LO), BI(6)},
    {X, Z, Y, MF(Z,LO), MF(Z,HI), IS(Y,NEG), IF(Y,HI), BI(6), BF(X,HI)},
    {X, Z, Y, MF(Z,LO), MC(Z,X,LO,POS), IF(Y,LO), IF(Y,HI), BF(X,LO), BI(6)},
    {X, Z, Y, MF(Z,LO), MC(Z,X,HI,POS), IS(Y,NEG), IF(Y,HI), BI(3), BF(X,HI)},
    {X, Z, Y, MF(Z,LO), MF(Z,HI), IS(Y,NEG), IF(Y,HI), BF(X,LO), BI(3)},
    {X, Z, Y, MF(Z,LO), MC(Z,X,HI,NEG), IF(Y,LO), IS(Y,POS), BI(3), BF(X,HI)},
    {X, Z, Y, MF(Z,LO), MF(Z,HI), IF(Y,LO), IS(Y,POS), BF(X,LO), BI(3)},
    {X, Z, Y, MC(Z,X,HI,NEG), MF(Z,HI), IF(Y,LO), IF(Y,HI), BI(3), BF(X,HI)},
    {X, Z, Y, MC(Z,X,HI,NEG), MF(Z,HI), IS(Y,NEG), IF(Y,HI), BI(7), BF(X,HI)},
    {X, Z, Y, MF(Z,LO), MF(Z,HI), IS(Y,NEG), IF(Y,HI), BF(X,LO), BI(7)},
    {X, Z, Y, MC(Z,X,HI,POS), MF(Z,HI), IF(Y,LO), IS(Y,POS), BI(7), BF(X,HI)},
    {X, Z, Y, MF(Z,LO), MF(Z,HI), IF(Y,LO), IS(Y,POS), BF(X,LO), BI(7)},
    {X, Z, Y, MF(Z,LO), MC(Z,X,HI,POS), IF(Y,LO), IF(Y,HI), BI(7), BF(X,HI)},
    {X, Z, Y, MF(Z,LO), MC(Z,X,HI,POS), IS(Y,NEG), IF(Y,HI), BF(X,LO), BI(3)},
    {X, Z, Y, MF(Z,LO), MF(Z,HI), IS(Y,NEG), IF(Y,HI), BI(3), BF(X,HI)},
    {X, Z, Y, MF(Z,LO), MC(Z,X,HI,NEG), IF(Y,LO), IS(Y,POS), BF(X,LO), BI(3)},
    {X, Z, Y, MF(Z,LO), MF(Z,HI), IF(Y,LO), IS(Y,POS), BI(3), BF(X,HI)},
    {X, Z, Y, MC(Z,X,HI,NEG), MF(Z,HI), IF(Y,LO), IF(Y,HI), BF(X,LO), BI(3)},
    {X, Z, Y, MC(Z,X,HI,NEG), MF(Z,HI), IS(Y,NEG), IF(Y,HI), BF(X,LO), BI(7)},
    {X, Z, Y, MF(Z,LO), MF(Z,HI), IS(Y,NEG), IF(Y,HI), BI(7), BF(X,HI)},
    {X, Z, Y, MC(Z,X,HI,POS), MF(Z,HI), IF(Y,LO), IS(Y,POS), BF(X,LO), BI(7)},
    {X, Z, Y, MF(Z,LO), MF(Z,HI), IF(Y,LO), IS(Y,POS), BI(7), BF(X,HI)},
    {X, Z, Y, MF(Z,LO), MC(Z,X,HI,POS), IF(Y,LO), IF(Y,HI), BF(X,LO), BI(7)},
    {Y, Z, X, MF(Z,LO), MF(Z,HI), IF(X,LO), IS(X,POS), BF(Y,LO), BF(Y,HI)},
    {Y, Z, X, MF(Z,LO), MF(Z,HI), IS(X,NEG), IF(X,HI), BF(Y,LO), BF(Y,HI)},
    {X, Z, Y, MF(Z,LO), MF(Z,HI), IF(Y,LO), IS(Y,POS), BF(X,LO), BF(X,HI)},
    {X, Z, Y, MF(Z,LO), MF(Z,HI), IS(Y,NEG), IF(Y,HI), BF(X,LO), BF(X,HI)},
    {X, Y, Z, MF(Y,LO), MF(Y,HI), IF(Z,LO), IS(Z,POS), BF(X,LO), BF(X,HI)},
    {X, Y, Z, MF(Y,LO), MF(Y,HI), IS(Z,NEG), IF(Z,HI), BF(X,LO), BF(X,HI)},
    {Z, Y, X, MF(Y,LO), MC(Y,Z,LO,POS), IF(X,LO), IS(X,POS), BN(3), BF(Z,HI)},
    {Z, Y, X, MF(Y,LO), MF(Y,HI), IF(X,LO), IS(X,POS), BF(Z,LO), BN(3)},
    {Z, Y, X, MF(Y,LO), MC(Y,Z,LO,NEG), IS(X,NEG), IF(X,HI), BN(3), BF(Z,HI)},
    {Z, Y, X, MF(Y,LO), MF(Y,HI), IS(X,NEG), IF(X,HI), BF(Z,LO), BN(3)},
    {Z, Y, X, MC(Y,Z,LO,NEG), MF(Y,HI), IF(X,LO), IF(X,HI), BN(3), BF(Z,HI)},
    {Z, Y, X, MF(Y,LO), MC(Y,Z,LO,POS), IF(X,LO), IS(X,POS), BF(Z,LO), BN(3)},
    {Z, Y, X, MF(Y,LO), MF(Y,HI), IF(X,LO), IS(X,POS), BN(3), BF(Z,HI)},
    {Z, Y, X, MF(Y,LO), MC(Y,Z,LO,NEG), IS(X,NEG), IF(X,HI), BF(Z,LO), BN(3)},
    {Z, Y, X, MF(Y,LO), MF(Y,HI), IS(X,NEG), IF(X,HI), BN(3), BF(Z,HI)},
    {Z, Y, X, MC(Y,Z,LO,NEG), MF(Y,HI), IF(X,LO), IF(X,HI), BF(Z,LO), BN(3)},
    {Z, Y, X, MC(Y,Z,LO,NEG), MF(Y,HI), IF(X,LO), IS(X,POS), BN(0), BF(Z,HI)},
    {Z, Y, X, MF(Y,LO), MF(Y,HI), IF(X,LO), IS(X,POS), BF(Z,LO), BN(0)},
    {Z, Y, X, MC(Y,Z,LO,POS), MF(Y,HI), IS(X,NEG), IF(X,HI), BN(0), BF(Z,HI)},
    {Z, Y, X, MF(Y,LO), MF(Y,HI), IS(X,NEG), IF(X,HI), BF(Z,LO), BN(0)},
    {Z, Y, X, MF(Y,LO), MC(Y,Z,LO,POS), IF(X,LO), IF(X,HI), BN(0), BF(Z,HI)},
    {Z, Y, X, MC(Y,Z,LO,NEG), MF(Y,HI), IF(X,LO), IS(X,POS), BF(Z,LO), BN(0)},
    {Z, Y, X, MF(Y,LO), MF(Y,HI), IF(X,LO), IS(X,POS), BN(0), BF(Z,HI)},
    {Z, Y, X, MC(Y,Z,LO,POS), MF(Y,HI), IS(X,NEG), IF(X,HI), BF(Z,LO), BN(0)},
    {Z, Y, X, MF(Y,LO), MF(Y,HI), IS(X,NEG), IF(X,HI), BN(0), BF(Z,HI)},
    {Z, Y, X, MF(Y,LO), MC(Y,Z,LO,POS), IF(X,LO), IF(X,HI), BF(Z,LO), BN(0)},
    {Z, Y, X, MF(Y,LO), MC(Y,Z,HI,POS), IS(X,NEG), IF(X,HI), BN(2), BF(Z,HI)},
    {Z, Y, X, MF(Y,LO), MF(Y,HI), IS(X,NEG), IF(X,HI), BF(Z,LO), BN(2)},
    {Z, Y, X, MF(Y,LO), MC(Y,Z,HI,NEG), IF(X,LO), IS(X,POS), BN(2), BF(Z,HI)},
    {Z, Y, X, MF(Y,LO), MF(Y,HI), IF(X,LO), IS(X,POS), BF(Z,LO), BN(2)},
    {Z, Y, X, MC(Y,Z,HI,NEG), MF(Y,HI), IF(X,LO), IF(X,HI), BN(2), BF(Z,HI)},
    {Z, Y, X, MF(Y,LO), MC(Y,Z,HI,POS), IS(X,NEG), IF(X,HI), BF(Z,LO), BN(2)},
    {Z, Y, X, MF(Y,LO), MF(Y,HI), IS(X,NEG), IF(X,HI), BN(2), BF(Z,HI)},
    {Z, Y, X, MF(Y,LO), MC(Y,Z,HI,NEG), IF(X,LO), IS(X,POS), BF(Z,LO), BN(2)},
    {Z, Y, X, MF(Y,LO), MF(Y,HI), IF(X,LO), IS(X,POS), BN(2), BF(Z,HI)},
    {Z, Y, X, MC(Y,Z,HI,NEG), MF(Y,HI), IF(X,LO), IF(X,HI), BF(Z,LO), BN(2)},
    {Z, Y, X, MC(Y,Z,HI,NEG), MF(Y,HI), IS(X,NEG), IF(X,HI), BN(1), BF(Z,HI)},
    {Z, Y, X, MF(Y,LO), MF(Y,HI), IS(X,NEG), IF(X,HI), BF(Z,LO), BN(1)},
    {Z, Y, X, MC(Y,Z,HI,POS), MF(Y,HI), IF(X,LO), IS(X,POS), BN(1), BF(Z,HI)},
    {Z, Y, X, MF(Y,LO), MF(Y,HI), IF(X,LO), IS(X,POS), BF(Z,LO), BN(1)},
    {Z, Y, X, MF(Y,LO), MC(Y,Z,HI,POS), IF(X,LO), IF(X,HI), BN(1), BF(Z,HI)},
    {Z, Y, X, MC(Y,Z,HI,NEG), MF(Y,HI), IS(X,NEG), IF(X,HI), BF(Z,LO), BN(1)},
    {Z, Y, X, MF(Y,LO), MF(Y,HI), IS(X,NEG), IF(X,HI), BN(1), BF(Z,HI)},
    {Z, Y, X, MC(Y,Z,HI,POS), MF(Y,HI), IF(X,LO), IS(X,POS), BF(Z,LO), BN(1)},
    {Z, Y, X, MF(Y,LO), MF(Y,HI), IF(X,LO), IS(X,POS), BN(1), BF(Z,HI)},
    {Z, Y, X, MF(Y,LO), MC(Y,Z,HI,POS), IF(X,LO), IF(X,HI), BF(Z,LO), BN(1)},
};

double t2_bound(const Bond& g, uint8_t code, const double ip[8], const double np[4]) {
    if (code < 8) return (code & 1) ? g.hi(code >> 1) : g.lo(code >> 1);
    if (code < 16) return ip[code - 8];
    return np[code - 16];
}

bool sign_ok(int8_t want, double v) { return want == 0 || (want > 0 ? v > 0.0 : v < 0.0); }

void type2(const Bond& g) {
    double ip[8] = {0, 0, 0, 0, 0, 0, 0, 0}, np[4] = {0, 0, 0, 0};
    const int b = eight_edges(g, ip);
    int nb = -1;
    for (const T2Rule& r : kT2Rules) {
        if (r.b != b) continue;
        if (r.nb >= 0) {
            if (nb < 0) nb = four_edges(g, np);
            if (nb != r.nb) continue;
        }
        if (r.cmp == 1 && !(ip[2] < ip[7])) continue;
        if (r.cmp == 2 && !(ip[3] < ip[6])) continue;
        if (!sign_ok(r.sx, g.xj[0]) || !sign_ok(r.sy, g.xj[1]) || !sign_ok(r.sz, g.xj[2])) continue;
        switch (r.kind) {
            case S1: t2_sub1(g, r.o, r.m, r.i); break;
            case S2: t2_sub2(g, r.o, r.m, r.i); break;
            case RS:
            case RD:
                for (int k = 0; k < r.count; ++k) {
                    const T2Reg& q = kT2Regs[r.first + k];
                    g.add(q.o, q.m, q.i, q.l0, q.l1, q.l2, q.l3, t2_bound(g, q.a, ip, np), t2_bound(g, q.b, ip, np),
                          r.kind == RD);
                }
                break;
            default: break;
        }
        return;
    }
}

// ---------------------------------------------------------------- bonds

// CalcBondForceIntg's classification (pdDataManager2.cpp:1227-1291): no force
// beyond the horizon, the whole cell (CalcConfigurationType3,
// pdIntgManager.cpp:3471-3482) inside it, else AdaptiveIntegration
// (pdIntgManager.cpp:523-546): type 1 on an axis through node i, else type 2.
void plan_bond(const Bond& g, double dmin, double dmax) {
    if (g.delta <= dmin) return;
    if (g.delta >= dmax) {
        g.add(X, Y, Z, face(Y, LO), face(Y, HI), face(Z, LO), face(Z, HI), g.lo(X), g.hi(X), true);
        return;
    }
    const bool a0 = g.xj[0] != 0.0, a1 = g.xj[1] != 0.0, a2 = g.xj[2] != 0.0;
    if ((a0 && !a1 && !a2) || (!a0 && a1 && !a2) || (!a0 && !a1 && a2)) type1(g);
    else type2(g);
}

Bond make_bond(const double* x, int64_t i, int64_t j, double dx, double delta, std::vector<pd_ai_region>* out) {
    Bond g;
    for (int a = 0; a < 3; ++a) g.xj[a] = x[3 * j + a] - x[3 * i + a];
    g.delta = delta;
    g.dx = dx;
    g.out = out;
    return g;
}

// entry of node j in the (ascending) row of node i, or -1
int64_t find_entry(const int64_t* row_ptr, const int32_t* col, int64_t i, int64_t j) {
    const int32_t* b = col + row_ptr[i];
    const int32_t* e = col + row_ptr[i + 1];
    const int32_t* p = std::lower_bound(b, e, (int32_t)j);
    return (p != e && *p == j) ? (int64_t)(p - col) : -1;
}

struct NoOp {
    void operator()(const double*, int, double* f) const { f[0] = f[1] = f[2] = 0.0; }
};

// records the global coordinates of the first `want` points
struct Record {
    const double* xi;
    std::vector<double>* pts;
    int64_t want;
    void operator()(const double* p, int, double* f) {
        f[0] = f[1] = f[2] = 0.0;
        if ((int64_t)pts->size() < 3 * want) {
            pts->push_back(p[0] + xi[0]);
            pts->push_back(p[1] + xi[1]);
            pts->push_back(p[2] + xi[2]);
        }
    }
};

}  // namespace

}  // namespace pdh

using pdh::make_bond;

extern "C" int pd_ai_plan(int64_t n, const double* coords, const int64_t* row_ptr, const int32_t* col, double dx,
                          double delta, int64_t* reg_ptr, pd_ai_region* regions, int64_t capacity,
                          int64_t* num_regions) {
    if (n < 0 || (n > 0 && (!coords || !row_ptr || !col)) || !(dx > 0.0) || !(delta > 0.0))
        return PD_ERR_ARG;
    std::vector<pd_ai_region> out;
    std::vector<int64_t> ptr((size_t)row_ptr[n] + 1, 0);
    for (int64_t i = 0; i < n; ++i) {
        for (int64_t p = row_ptr[i]; p < row_ptr[i + 1]; ++p) {
            const int64_t j = col[p];
            if (j < 0 || j >= n || j == i) return PD_ERR_ARG;
            // the bond was built by the lower node (InitBond, pdDataManager2.cpp:20-63):
            // its distances are from that node to the other's cell
            const int64_t lo = std::min(i, j), hi = std::max(i, j);
            double dmin, dmax;
            pdh::cube_distance(coords + 3 * lo, coords + 3 * hi, dx, &dmin, &dmax);
            pdh::plan_bond(make_bond(coords, i, j, dx, delta, &out), dmin, dmax);
            ptr[p + 1] = (int64_t)out.size();
        }
    }
    if (num_regions) *num_regions = (int64_t)out.size();
    if (reg_ptr) std::copy(ptr.begin(), ptr.end(), reg_ptr);
    if (!regions) return PD_OK;
    if (capacity < (int64_t)out.size()) return PD_ERR_CAPACITY;
    std::copy(out.begin(), out.end(), regions);
    return PD_OK;
}

extern "C" int pd_ai_mls_table(int64_t n, const double* coords, const int64_t* row_ptr, const int32_t* col,
                               const int64_t* reg_ptr, const pd_ai_region* regions, double dx, double delta,
                               int trap, const int64_t* cb_ptr, const int32_t* cb_idx, double rw, int64_t* tab_ptr,
                               double* tab_coeff, int64_t capacity, int64_t* num_coeff, int64_t* bad_node) {
    if (n < 0 || (n > 0 && (!coords || !row_ptr || !col || !reg_ptr || !cb_ptr || !cb_idx || !tab_ptr)) ||
        trap < 1 || trap > 3 || !(rw > 0.0))
        return PD_ERR_ARG;
    // node j's list: the points of the bonds i -> j for i over j's family in
    // ascending order (the setup pass visits node i, then its family), all of
    // each bond's regions in order; the force pass reads entry k for a
    // region's k-th point, so K_j = the most points any region of a bond to j
    // evaluates
    std::vector<int64_t> K((size_t)n, 0);
    std::vector<int64_t> src((size_t)row_ptr[n], -1);  // entry i -> j for entry j -> i
    for (int64_t j = 0; j < n; ++j) {
        int64_t total = 0;
        for (int64_t q = row_ptr[j]; q < row_ptr[j + 1]; ++q) {
            const int64_t i = col[q];
            const int64_t p = pdh::find_entry(row_ptr, col, i, j);
            if (p < 0) return PD_ERR_ARG;  // the family is not symmetric
            src[q] = p;
            pdh::Bond g = make_bond(coords, i, j, dx, delta, nullptr);
            pdh::NoOp none;
            for (int64_t r = reg_ptr[p]; r < reg_ptr[p + 1]; ++r) {
                double f[3];
                const int c = pd_ai::region(regions[r], trap, g.xj, delta, dx, none, f);
                K[j] = std::max<int64_t>(K[j], c);
                total += c;
            }
        }
        (void)total;
    }
    tab_ptr[0] = 0;
    int64_t ncoef = 0;
    for (int64_t j = 0; j < n; ++j) {
        tab_ptr[j + 1] = tab_ptr[j] + K[j];
        ncoef += K[j] * (cb_ptr[j + 1] - cb_ptr[j]);
    }
    if (num_coeff) *num_coeff = ncoef;
    if (!tab_coeff) return PD_OK;
    if (capacity < ncoef) return PD_ERR_CAPACITY;
    std::vector<int64_t> coff((size_t)n + 1, 0);
    for (int64_t j = 0; j < n; ++j) coff[j + 1] = coff[j] + K[j] * (cb_ptr[j + 1] - cb_ptr[j]);
    std::atomic<int64_t> next(0), bad(-1);
    auto worker = [&]() {
        std::vector<double> pts, pw;
        for (;;) {
            const int64_t j = next.fetch_add(1);
            if (j >= n || bad.load() >= 0) return;
            if (K[j] == 0) continue;
            pts.clear();
            for (int64_t q = row_ptr[j]; q < row_ptr[j + 1] && (int64_t)pts.size() < 3 * K[j]; ++q) {
                const int64_t i = col[q], p = src[q];
                pdh::Bond g = make_bond(coords, i, j, dx, delta, nullptr);
                pdh::Record rec{coords + 3 * i, &pts, K[j]};
                for (int64_t r = reg_ptr[p]; r < reg_ptr[p + 1] && (int64_t)pts.size() < 3 * K[j]; ++r) {
                    double f[3];
                    pd_ai::region(regions[r], trap, g.xj, delta, dx, rec, f);
                }
            }
            const int64_t nc = cb_ptr[j + 1] - cb_ptr[j];
            pw.resize((size_t)nc * 11);
            for (int64_t k = 0; k < K[j]; ++k) {
                if (!pdh::mls_point(coords, cb_idx + cb_ptr[j], nc, &pts[3 * k], rw, pw.data(),
                                    tab_coeff + coff[j] + k * nc)) {
                    int64_t e = -1;
                    bad.compare_exchange_strong(e, j);
                    return;
                }
            }
        }
    };
    unsigned nt = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    for (unsigned t = 1; t < nt; ++t) pool.emplace_back(worker);
    worker();
    for (auto& th : pool) th.join();
    if (bad.load() >= 0) {
        if (bad_node) *bad_node = bad.load();
        return PD_ERR_SINGULAR;
    }
    return PD_OK;
}
