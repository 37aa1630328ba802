// FP32-compensated form of the bond force and the MLS gather.
//
// Compiled with -ftz=true -prec-div=false -prec-sqrt=false: reciprocals and
// reciprocal square roots are single MUFU operations.
//
// Numerics.  The stretch of a bond is tiny (1e-6..1e-3) next to its length,
// so (|xi+eta| - |xi|) / |xi| loses every digit in FP32.  The kernel never
// forms that difference: with d = |xi+eta|^2 - |xi|^2 = eta.(2 xi + eta),
//     s = d / (r (p + r)),   f = c beta s (xi+eta) / p,
// every term is accurate to FP32 rounding relative to the strain itself.
// eta is assembled from differences that are exact or nearly so:
//     eta = (us_j - u_i) + (ug_j,g - us_j)
// where the second term is produced by the gather directly, and the first is
// (hi_j - hi_i) + (lo_j - lo_i) from FP32 hi/lo splits of the FP64 values
// (hi = fl32(u), lo = fl32(u - hi)); hi_j - hi_i is exact whenever the two
// are within a factor of two (Sterbenz), which is the case for neighbours
// unless both are tiny.  Coordinates are split the same way.  Per-bond forces
// are summed in FP32 over the Gauss points, the family sum of each node is
// Kahan-compensated, and the state update stays FP64.
#include <algorithm>
#include <climits>

#include "pd_internal.cuh"
#include "pd_stage.cuh"

namespace pd {

namespace {

inline unsigned blocks_for(int64_t n, int bs) { return (unsigned)((n + bs - 1) / bs); }

__device__ __forceinline__ double time_factor(const BcDev& b, double t) {
    if (b.type == PD_BC_VELOC) return (t <= b.end_time) ? 1.0 : 0.0;
    if (b.load_type == 1.0) return (t <= b.end_time) ? t / b.end_time : 1.0;
    return 1.0;
}

__device__ __forceinline__ float4 ld4(const float* p) { return __ldg(reinterpret_cast<const float4*>(p)); }

// data the same launch rewrites (the persistent kernel): through L2, never a
// possibly stale L1 line; read-only data keep the non-coherent path
template <bool PERSIST>
__device__ __forceinline__ float4 ld4m(const float* p) {
    return PERSIST ? __ldcg(reinterpret_cast<const float4*>(p)) : __ldg(reinterpret_cast<const float4*>(p));
}
template <bool PERSIST>
__device__ __forceinline__ double ldm(const double* p) {
    return PERSIST ? __ldcg(p) : __ldg(p);
}

struct PointF {
    float hx, hy, hz, W, A, B;  // offset of the point from its node, weight*vol/8, beta = sat((A - r) B)
};

template <int NPT>
struct PointPack {
    PointF p[NPT > 0 ? NPT : 1];
};

// FP32 operations with explicit rounding (round to nearest, denormals
// flushed, never contracted), written once so that the scalar and the packed
// code paths below round identically
__device__ __forceinline__ float fadd(float a, float b) {
    float d;
    asm("add.rn.ftz.f32 %0, %1, %2;" : "=f"(d) : "f"(a), "f"(b));
    return d;
}
__device__ __forceinline__ float fmul(float a, float b) {
    float d;
    asm("mul.rn.ftz.f32 %0, %1, %2;" : "=f"(d) : "f"(a), "f"(b));
    return d;
}
__device__ __forceinline__ float ffma(float a, float b, float c) {
    float d;
    asm("fma.rn.ftz.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}

// Two FP32 values in one 64-bit register, and sm_100's packed FP32
// arithmetic on them (one instruction for both lanes, each lane rounded as
// the scalar operation above rounds)
typedef unsigned long long f2;
__device__ __forceinline__ f2 f2_make(float lo, float hi) {
    f2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void f2_split(f2 v, float& lo, float& hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ f2 f2_add(f2 a, f2 b) {
    f2 d;
    asm("add.rn.ftz.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f2 f2_mul(f2 a, f2 b) {
    f2 d;
    asm("mul.rn.ftz.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f2 f2_fma(f2 a, f2 b, f2 c) {
    f2 d;
    asm("fma.rn.ftz.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}

// ---- per-point force of the FP32 form ----
//
// For a bond vector x (cell j's Gauss point minus node i) and relative
// displacement e, with y = x + e, r = |x|, p = |y| and dd = p^2 - r^2 =
// e.(2x + e) = e.(x + y), the point force of pdDataManager2.cpp:1320-1343 is
//     f = W beta(r) s y / p,   s = (p - r) / r,
// and W beta s / p = K h(eps) with K = W beta(r) / r and eps = dd / r^2:
//     h(eps) = dd / ((p + r) p) = 1 - (1 + eps)^(-1/2).
// K and 1/r^2 depend on the bond's lattice offset and the point only (pt_geo),
// so the lattice kernels can take them from a table.  For |eps| < 1/64,
// h is the binomial series eps (1/2 - 3/8 eps + 5/16 eps^2 - 35/128 eps^3),
// whose truncation error is below 0.5 eps^4 relative (3e-8 at the bound, under
// half an FP32 ulp); strains of 1e-5..1e-3 give eps of 2e-5..2e-3.  Larger
// |eps| takes the exact form dd / ((p + r) p) with reciprocal square roots.
// Every operation is written with an explicit rounding intrinsic, so that the
// scalar kernels and the packed (two points per instruction) stencil kernel
// round alike, and the forces of the eight points of a bond are summed in
// two chains, the even points and the odd points, added at the end.
// The critical-stretch test s > ecrit reads eps > ecrit (2 + ecrit).
constexpr float kSeriesMax = 1.0f / 64.0f;
constexpr float kH1 = 0.5f, kH2 = -0.375f, kH3 = 0.3125f, kH4 = -0.2734375f;

__device__ __forceinline__ void pt_geo(const PointF& P, float x0, float x1, float x2, float& K, float& r2inv) {
    const float r2 = ffma(x0, x0, ffma(x1, x1, fmul(x2, x2)));
    const float rinv = rsqrtf(r2);
    const float r = fmul(r2, rinv);
    const float beta = __saturatef(fmul(fadd(P.A, -r), P.B));
    K = fmul(fmul(P.W, beta), rinv);
    r2inv = fmul(rinv, rinv);
}

__device__ __forceinline__ float pt_series(float eps) {
    float c = ffma(eps, kH4, kH3);
    c = ffma(eps, c, kH2);
    c = ffma(eps, c, kH1);
    return fmul(eps, c);
}

__device__ __forceinline__ float pt_exact(float x0, float x1, float x2, float dd) {
    const float r2 = ffma(x0, x0, ffma(x1, x1, fmul(x2, x2)));
    const float p2 = fadd(r2, dd);
    const float pinv = rsqrtf(p2), rinv = rsqrtf(r2);
    const float p = fmul(p2, pinv), r = fmul(r2, rinv);
    return fmul(fmul(dd, pinv), __frcp_rn(fadd(p, r)));
}

// one point: F (three components of its chain) += f
template <bool HASFAIL>
__device__ __forceinline__ void pt_force(float x0, float x1, float x2, float K, float r2inv, float e0, float e1,
                                         float e2, float epsc, float* F) {
    const float y0 = fadd(x0, e0), y1 = fadd(x1, e1), y2 = fadd(x2, e2);
    const float dd = ffma(e0, fadd(x0, y0), ffma(e1, fadd(x1, y1), fmul(e2, fadd(x2, y2))));
    const float eps = fmul(dd, r2inv);
    const float h = fabsf(eps) < kSeriesMax ? pt_series(eps) : pt_exact(x0, x1, x2, dd);
    float fm = fmul(K, h);
    if (HASFAIL && eps > epsc) fm = 0.f;
    F[0] = ffma(fm, y0, F[0]);
    F[1] = ffma(fm, y1, F[1]);
    F[2] = ffma(fm, y2, F[2]);
}

// The same for two points at once (lo and hi lanes), lane by lane the
// operations of pt_force; a lane outside the series range takes pt_exact.
// SERIES: the series form only, with no branch to the exact form (so the
// point chains of a bond interleave freely); a lane outside the series range
// sets *wide, and the caller discards the result and evaluates again without
// SERIES.
template <bool HASFAIL, bool SERIES = false>
__device__ __forceinline__ void pt_force2(f2 x0, f2 x1, f2 x2, f2 K, f2 r2inv, f2 e0, f2 e1, f2 e2, float epsc,
                                          f2* F, bool* wide = nullptr) {
    const f2 y0 = f2_add(x0, e0), y1 = f2_add(x1, e1), y2 = f2_add(x2, e2);
    const f2 dd = f2_fma(e0, f2_add(x0, y0), f2_fma(e1, f2_add(x1, y1), f2_mul(e2, f2_add(x2, y2))));
    const f2 eps = f2_mul(dd, r2inv);
    f2 c = f2_fma(eps, f2_make(kH4, kH4), f2_make(kH3, kH3));
    c = f2_fma(eps, c, f2_make(kH2, kH2));
    c = f2_fma(eps, c, f2_make(kH1, kH1));
    f2 h = f2_mul(eps, c);
    float el, eh;
    f2_split(eps, el, eh);
    if (SERIES) {
        *wide = *wide | !(fabsf(el) < kSeriesMax) | !(fabsf(eh) < kSeriesMax);
    } else if (!(fabsf(el) < kSeriesMax) || !(fabsf(eh) < kSeriesMax)) {
        float hl, hh, dl, dh, a0, b0, a1, b1, a2, b2;
        f2_split(h, hl, hh);
        f2_split(dd, dl, dh);
        f2_split(x0, a0, b0);
        f2_split(x1, a1, b1);
        f2_split(x2, a2, b2);
        if (!(fabsf(el) < kSeriesMax)) hl = pt_exact(a0, a1, a2, dl);
        if (!(fabsf(eh) < kSeriesMax)) hh = pt_exact(b0, b1, b2, dh);
        h = f2_make(hl, hh);
    }
    f2 fm = f2_mul(K, h);
    if (HASFAIL) {
        float fl, fh;
        f2_split(fm, fl, fh);
        if (el > epsc) fl = 0.f;
        if (eh > epsc) fh = 0.f;
        fm = f2_make(fl, fh);
    }
    F[0] = f2_fma(fm, y0, F[0]);
    F[1] = f2_fma(fm, y1, F[1]);
    F[2] = f2_fma(fm, y2, F[2]);
}

// eps above which a bond has failed: s > ecrit  <=>  eps > ecrit (2 + ecrit)
__device__ __forceinline__ float eps_crit(float ecrit) { return fmul(ecrit, fadd(2.0f, ecrit)); }

// us_j - u_i from FP32 hi/lo splits
__device__ __forceinline__ float split_diff(float jh, float jl, float ih, float il) {
    return fadd(fadd(jh, -ih), fadd(jl, -il));
}

// Four Gauss points q..q+3 of cell j on one bond (without the pair
// coefficient), given xi_ij (dx), us_j - u_i (du) and the Gauss-point
// displacements of j relative to us_j (u4: x[4], y[4], z[4]).  F[0..2] is the
// chain of the even points, F[3..5] that of the odd points.
template <bool HASFAIL>
__device__ __forceinline__ void bond4(const PointPack<8>& G, int q, const float* u4, const float* dx,
                                      const float* du, float epsc, float* F) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const PointF& P = G.p[q + k];
        const float x0 = fadd(dx[0], P.hx), x1 = fadd(dx[1], P.hy), x2 = fadd(dx[2], P.hz);
        float K, r2inv;
        pt_geo(P, x0, x1, x2, K, r2inv);
        const float e0 = fadd(du[0], u4[k]), e1 = fadd(du[1], u4[4 + k]), e2 = fadd(du[2], u4[8 + k]);
        pt_force<HASFAIL>(x0, x1, x2, K, r2inv, e0, e1, e2, epsc, F + 3 * (k & 1));
    }
}

// the bond force of the two chains
__device__ __forceinline__ void chains_sum(const float* F6, float* F) {
    F[0] = fadd(F6[0], F6[3]);
    F[1] = fadd(F6[1], F6[4]);
    F[2] = fadd(F6[2], F6[5]);
}

struct Own {
    float uh[3], ul[3];  // displacement of the node, FP32 hi/lo
    float ph[3], pl[3];  // position hi/lo (off the lattice path)
    int lat;             // packed lattice position
    float be, sf, c, e;
    int mat;
    float s[3], k[3];    // Kahan sum of the family force
};

// the bond force F c added to the family sum (products rounded on their own,
// never contracted into the subtraction, so every kernel rounds alike)
__device__ __forceinline__ void kahan_add(Own& o, const float* F, float c) {
    const float F0 = __fmul_rn(F[0], c), F1 = __fmul_rn(F[1], c), F2 = __fmul_rn(F[2], c);
    float y = F0 - o.k[0], t = o.s[0] + y;
    o.k[0] = (t - o.s[0]) - y;
    o.s[0] = t;
    y = F1 - o.k[1]; t = o.s[1] + y; o.k[1] = (t - o.s[1]) - y; o.s[1] = t;
    y = F2 - o.k[2]; t = o.s[2] + y; o.k[2] = (t - o.s[2]) - y; o.s[2] = t;
}

template <bool LAT, bool BDRY, bool SFAC, bool MULTIMAT, bool PERSIST = false>
__device__ __forceinline__ void load_own(const Dev& d, int64_t i, Own& o) {
    const int64_t N = d.n;
    const double* src = d.bc[i] >= 0 ? d.U : d.us;
    for (int a = 0; a < 3; ++a) {
        const double u = PERSIST ? __ldcg(src + a * N + i) : src[a * N + i];
        o.uh[a] = (float)u;
        o.ul[a] = (float)(u - (double)o.uh[a]);
        o.s[a] = o.k[a] = 0.f;
    }
    const float* sb = d.sblk + 8 * i;
    if (LAT) {
        o.lat = d.lat[i];
    } else {
        for (int a = 0; a < 3; ++a) {
            o.ph[a] = sb[a];
            o.pl[a] = sb[3 + a];
        }
    }
    o.be = BDRY ? sb[6] : 1.f;
    o.sf = SFAC ? sb[7] : 1.f;
    o.mat = MULTIMAT ? d.mat[i] : 0;
    o.c = MULTIMAT ? (float)d.mats[o.mat].spring : d.c0;
    o.e = MULTIMAT ? (float)d.mats[o.mat].ecrit : d.e0;
}

// vbuf_i = vbase_i + (F_i + n_bonds rho g) dt_s / rho; vbase is vbuf itself,
// or V at the first stage of a persistent step (InitDynamicSolve's vbuf = V)
template <bool PERSIST = false>
__device__ __forceinline__ void store_own(const Dev& d, int64_t i, const Own& o, int64_t nbonds, double dts,
                                          const double* vbase) {
    const int64_t N = d.n;
    const MatDev& M = d.mats[o.mat];
    const double rho = M.density;
    for (int a = 0; a < 3; ++a) {
        const double v0 = PERSIST ? __ldcg(vbase + a * N + i) : vbase[a * N + i];
        d.vbuf[a * N + i] = v0 + ((double)o.s[a] - (double)o.k[a] + (double)nbonds * (M.grav[a] * rho)) * dts / rho;
    }
}

// FGI with 2x2x2 Gauss points, two nodes per thread.  The work order pairs
// x-adjacent nodes; the thread walks the merge of their two ascending family
// lists and loads every neighbour's block once for both bonds, which cuts
// the L1 traffic per evaluation (the bound of this kernel) by the overlap of
// the two families.  pdDataManager.cpp:1917-1962 in FP32 form.
// Node blocks staged in shared memory (the tiled kernel): a box of the
// lattice [lo, lo + (lx, ly, ...)) with kTileStride floats per node.
constexpr int kSell = 16;        // nodes per SELL slice of the gather
constexpr int kTileStride = 36;  // 144 B: 16-byte aligned, and lanes reading
                                 // different nodes spread over the banks
struct SmemTile {
    const float* base;
    int lox, loy, loz, lx, ly;
};

// Nodes ia and ib (ib may be -1).  PERSIST (inside the persistent kernel)
// adds what the separate launches of a step do around the force: at the
// first stage u1 = us = U and vbuf starts from V; after the force the stage
// epilogue of both nodes at time t.  SMEM: neighbour blocks from a staged
// tile T instead of global memory.
template <bool HASFAIL, bool LAT, bool BDRY, bool SFAC, bool MULTIMAT, bool PERSIST, bool SMEM>
__device__ __forceinline__ void force_nodes(const Dev& d, const PointPack<8>& G, double dts, int64_t ia, int64_t ib,
                                            int pstage, double dt, double t, const SmemTile& T) {
    const int64_t N = d.n;
    if (PERSIST && pstage == 1) {
        for (int a = 0; a < 3; ++a) {
            const double ua = __ldcg(d.U + a * N + ia);
            d.u1[a * N + ia] = ua;
            d.us[a * N + ia] = ua;
            if (ib >= 0) {
                const double ub = __ldcg(d.U + a * N + ib);
                d.u1[a * N + ib] = ub;
                d.us[a * N + ib] = ub;
            }
        }
    }
    Own A, B;
    load_own<LAT, BDRY, SFAC, MULTIMAT, PERSIST>(d, ia, A);
    if (ib >= 0) load_own<LAT, BDRY, SFAC, MULTIMAT, PERSIST>(d, ib, B);
    int64_t pa = d.arow[ia], ea = d.arow[ia + 1];
    int64_t pb = 0, eb = 0;
    if (ib >= 0) {
        pb = d.arow[ib];
        eb = d.arow[ib + 1];
    }
    const int64_t nba = ea - pa, nbb = eb - pb;
    const float h = (float)d.dx;
    for (;;) {
        const int ja = pa < ea ? d.acol[pa] : INT_MAX;
        const int jb = pb < eb ? d.acol[pb] : INT_MAX;
        const int j = min(ja, jb);
        if (j == INT_MAX) break;
        int lj = 0;
        if (LAT) lj = d.lat[j];
        const float* bj = SMEM ? T.base + kTileStride * (((lj & 2047) - T.lox) +
                                                         T.lx * ((((lj >> 11) & 2047) - T.loy) +
                                                                 T.ly * ((lj >> 22) - T.loz)))
                               : d.nblk + (int64_t)j * 32;
        // hi0 hi1 hi2 lo0 | lo1 lo2 - -
        const float4 us0 = SMEM ? *reinterpret_cast<const float4*>(bj + 24) : ld4m<PERSIST>(bj + 24);
        const float4 us1 = SMEM ? *reinterpret_cast<const float4*>(bj + 28) : ld4m<PERSIST>(bj + 28);
        float pj[6];
        if (!LAT) {
            const float4 s0 = ld4(d.sblk + 8 * (int64_t)j), s1 = ld4(d.sblk + 8 * (int64_t)j + 4);
            pj[0] = s0.x; pj[1] = s0.y; pj[2] = s0.z; pj[3] = s0.w; pj[4] = s1.x; pj[5] = s1.y;
        }
        float bej = 1.f, sfj = 1.f;
        if (BDRY || SFAC) {
            const float2 v = __ldg(reinterpret_cast<const float2*>(d.sblk + 8 * (int64_t)j + 6));
            bej = v.x;
            sfj = v.y;
        }
        float cj = 0.f, ej = 0.f;
        if (MULTIMAT) {
            const int mj = d.mat[j];
            cj = (float)d.mats[mj].spring;
            ej = (float)d.mats[mj].ecrit;
        }
        const float ujh[3] = {us0.x, us0.y, us0.z}, ujl[3] = {us0.w, us1.x, us1.y};
        const bool has[2] = {ja == j, jb == j};
        // per-bond terms of both sides
        float dx[2][3], du[2][3], coef[2], ecrit[2];
#pragma unroll
        for (int side = 0; side < 2; ++side) {
            const Own& O = side == 0 ? A : B;
            if (LAT) {
                dx[side][0] = __fmul_rn((float)((lj & 2047) - (O.lat & 2047)), h);
                dx[side][1] = __fmul_rn((float)(((lj >> 11) & 2047) - ((O.lat >> 11) & 2047)), h);
                dx[side][2] = __fmul_rn((float)((lj >> 22) - (O.lat >> 22)), h);  // packed values are non-negative
            } else {
                for (int a = 0; a < 3; ++a) dx[side][a] = (pj[a] - O.ph[a]) + (pj[3 + a] - O.pl[a]);
            }
            for (int a = 0; a < 3; ++a) du[side][a] = split_diff(ujh[a], ujl[a], O.uh[a], O.ul[a]);
            float c = O.c;
            ecrit[side] = O.e;
            if (MULTIMAT) {
                c = fminf(c, cj);
                ecrit[side] = fminf(ecrit[side], ej);
            }
            if (BDRY) c *= 0.5f * (O.be + bej);
            if (SFAC) c *= 0.5f * (O.sf + sfj);
            coef[side] = c;
        }
        float F[2][6] = {{0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f, 0.f, 0.f}};
        const float epsc[2] = {HASFAIL ? eps_crit(ecrit[0]) : 0.f, HASFAIL ? eps_crit(ecrit[1]) : 0.f};
        // the eight Gauss points of cell j in two halves of four, each half
        // applied to both bonds
#pragma unroll
        for (int q = 0; q < 8; q += 4) {
            const float4 vx = SMEM ? *reinterpret_cast<const float4*>(bj + q) : ld4m<PERSIST>(bj + q);
            const float4 vy = SMEM ? *reinterpret_cast<const float4*>(bj + 8 + q) : ld4m<PERSIST>(bj + 8 + q);
            const float4 vz = SMEM ? *reinterpret_cast<const float4*>(bj + 16 + q) : ld4m<PERSIST>(bj + 16 + q);
            const float u4[12] = {vx.x, vx.y, vx.z, vx.w, vy.x, vy.y, vy.z, vy.w, vz.x, vz.y, vz.z, vz.w};
#pragma unroll
            for (int side = 0; side < 2; ++side)
                if (has[side])
                    bond4<HASFAIL>(G, q, u4, dx[side], du[side], epsc[side], F[side]);
        }
        if (has[0]) {
            float Fb[3];
            chains_sum(F[0], Fb);
            kahan_add(A, Fb, coef[0]);
            ++pa;
        }
        if (has[1]) {
            float Fb[3];
            chains_sum(F[1], Fb);
            kahan_add(B, Fb, coef[1]);
            ++pb;
        }
    }
    const double* vbase = (PERSIST && pstage == 1) ? d.V : d.vbuf;
    store_own<PERSIST>(d, ia, A, nba, dts, vbase);
    if (ib >= 0) store_own<PERSIST>(d, ib, B, nbb, dts, vbase);
    if (PERSIST) {
        stage_epilogue<false>(d, ia, pstage, dts, dt, t);
        if (ib >= 0) stage_epilogue<false>(d, ib, pstage, dts, dt, t);
    }
}

// the pair of work-order slots t2, t2 + 1
template <bool HASFAIL, bool LAT, bool BDRY, bool SFAC, bool MULTIMAT, bool PERSIST>
__device__ __forceinline__ void force_pair(const Dev& d, const PointPack<8>& G, double dts, int64_t t2, int pstage,
                                           double dt, double t) {
    const int64_t ia = d.order[t2];
    const int64_t ib = (t2 + 1 < d.n) ? d.order[t2 + 1] : -1;
    force_nodes<HASFAIL, LAT, BDRY, SFAC, MULTIMAT, PERSIST, false>(d, G, dts, ia, ib, pstage, dt, t, SmemTile{});
}

template <bool HASFAIL, bool LAT, bool BDRY, bool SFAC, bool MULTIMAT>
__global__ void __launch_bounds__(128, 4) k_force_f32c_pair(Dev d, PointPack<8> G, double dts) {
    const int64_t t2 = 2 * (blockIdx.x * (int64_t)blockDim.x + threadIdx.x);
    if (t2 >= d.n) return;
    force_pair<HASFAIL, LAT, BDRY, SFAC, MULTIMAT, false>(d, G, dts, t2, 0, 0.0, 0.0);
}

// Four nodes per thread: the work-order slots t4 .. t4+3 (x-adjacent in a
// node order whose tiles are at least four nodes wide) walk the merge of their
// four ascending family lists, so a neighbour block loaded once serves up to
// four bonds (the pair kernel: two).  Nodes on one lattice, one material, no
// failure test.  Per node the same arithmetic in the same order as
// k_force_f32c_pair, so the same result bit for bit.
template <bool BDRY, bool SFAC>
__global__ void __launch_bounds__(128, 3) k_force_f32c_quad(Dev d, PointPack<8> G, double dts) {
    const int64_t N = d.n;
    const int64_t t4 = 4 * (blockIdx.x * (int64_t)blockDim.x + threadIdx.x);
    if (t4 >= N) return;
    int64_t id[4], p[4], e[4], nb[4];
    Own O[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        id[k] = (t4 + k < N) ? d.order[t4 + k] : -1;
        p[k] = e[k] = 0;
        if (id[k] >= 0) {
            load_own<true, BDRY, SFAC, false>(d, id[k], O[k]);
            p[k] = d.arow[id[k]];
            e[k] = d.arow[id[k] + 1];
        }
        nb[k] = e[k] - p[k];
    }
    const float h = (float)d.dx;
    for (;;) {
        int js[4];
        int j = INT_MAX;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            js[k] = p[k] < e[k] ? d.acol[p[k]] : INT_MAX;
            j = min(j, js[k]);
        }
        if (j == INT_MAX) break;
        const float* bj = d.nblk + (int64_t)j * 32;
        const float4 us0 = ld4(bj + 24), us1 = ld4(bj + 28);  // hi0 hi1 hi2 lo0 | lo1 lo2 - -
        const int lj = d.lat[j];
        float bej = 1.f, sfj = 1.f;
        if (BDRY || SFAC) {
            const float2 v = __ldg(reinterpret_cast<const float2*>(d.sblk + 8 * (int64_t)j + 6));
            bej = v.x;
            sfj = v.y;
        }
        const float ujh[3] = {us0.x, us0.y, us0.z}, ujl[3] = {us0.w, us1.x, us1.y};
        float dx[4][3], du[4][3], coef[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            dx[k][0] = __fmul_rn((float)((lj & 2047) - (O[k].lat & 2047)), h);
            dx[k][1] = __fmul_rn((float)(((lj >> 11) & 2047) - ((O[k].lat >> 11) & 2047)), h);
            dx[k][2] = __fmul_rn((float)((lj >> 22) - (O[k].lat >> 22)), h);
            for (int a = 0; a < 3; ++a) du[k][a] = split_diff(ujh[a], ujl[a], O[k].uh[a], O[k].ul[a]);
            float c = O[k].c;
            if (BDRY) c *= 0.5f * (O[k].be + bej);
            if (SFAC) c *= 0.5f * (O[k].sf + sfj);
            coef[k] = c;
        }
        float F[4][6] = {};
#pragma unroll
        for (int q = 0; q < 8; q += 4) {
            const float4 vx = ld4(bj + q), vy = ld4(bj + 8 + q), vz = ld4(bj + 16 + q);
            const float u4[12] = {vx.x, vx.y, vx.z, vx.w, vy.x, vy.y, vy.z, vy.w, vz.x, vz.y, vz.z, vz.w};
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (js[k] == j) bond4<false>(G, q, u4, dx[k], du[k], 0.f, F[k]);
        }
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (js[k] == j) {
                float Fb[3];
                chains_sum(F[k], Fb);
                kahan_add(O[k], Fb, coef[k]);
                ++p[k];
            }
    }
#pragma unroll
    for (int k = 0; k < 4; ++k)
        if (id[k] >= 0) store_own<false>(d, id[k], O[k], nb[k], dts, d.vbuf);
}

// ------------------------------------------------------- lattice stencil
//
// On a complete box lattice the family of a node is a subset of one stencil
// S of lattice offsets.  The stencil kernel walks a bit mask of the family
// over the union list U2 = S u (S + e_x) of an x-adjacent node pair instead
// of two column lists, takes the bond vector from the offset, and reads the
// node blocks chunk-major, so that the 16 pairs of a warp row read a
// neighbour chunk from 1 KB of contiguous memory (8 lines instead of 32).
// Per node the same bond4 arithmetic in the same ascending neighbour order
// as the pair kernel's lattice variants: the same result bit for bit.
// (A first table of the geometric terms in global memory, read one float4
// per point, was slower than computing them: a warp-wide broadcast from L1
// still costs a wavefront per load.  The table below lives in shared memory,
// holds only what the series form needs, and serves two points per load.)

// One thread per x-adjacent node pair (A, B = A + 1) of a lattice row; a
// block covers tw pairs x (sten_by 16 / tw) rows x sten_bz layers (tw =
// sten_tw: 16, or 8 / 4 for narrow boxes).  A warp walks the
// union of its threads' masks over U2 in ascending offset (= ascending
// neighbour id for every thread), so the U2 entry and the table row are the
// same for the whole warp; a thread takes the bonds its own masks hold.
// Geometry per (entry, side, point pair) comes from the table of pt_geo
// values staged in shared memory (sten_tab, 16 bytes per two points: one
// broadcast load), and the eight points of a bond are evaluated two per
// packed instruction (pt_force2: the even point in the low lane, the odd in
// the high lane, which are the two chains of bond4).  Per node the same
// operations in the same order as bond4 on the lattice path: the same
// result bit for bit as the pair, quad and tiled kernels.
// One U2 entry of the pair (A, B): SIDES bit 0 = node A holds the bond,
// bit 1 = node B holds it.  Compiled for both sides together (the lattice
// interior, where the sides' independent chains interleave) and for each
// side alone.
template <bool HASFAIL, bool BDRY, bool SFAC, int SIDES, bool SERIES>
__device__ __forceinline__ void sten_entry(const Dev& d, int u, int64_t ia, int NX, int64_t NXY, const f2* hx,
                                           const f2* hy, const f2* hz, const float* epsc, float h, Own& A, Own& B,
                                           bool& wide) {
    const int64_t N = d.n;
    const float4* __restrict__ blk = reinterpret_cast<const float4*>(d.nblk);
    const int4 E = __ldg(d.sten_u2 + u);  // (id offset in one box), ox, oy, oz from A
    const int64_t j = ia + E.y + (int64_t)NX * E.z + NXY * E.w;
    const float4 us0 = __ldg(blk + 6 * N + j), us1 = __ldg(blk + 7 * N + j);  // hi0 hi1 hi2 lo0 | lo1 lo2 - -
    float bej = 1.f, sfj = 1.f;
    if (BDRY || SFAC) {
        const float2 v = __ldg(reinterpret_cast<const float2*>(d.sblk + 8 * j + 6));
        bej = v.x;
        sfj = v.y;
    }
    const float ujh[3] = {us0.x, us0.y, us0.z}, ujl[3] = {us0.w, us1.x, us1.y};
    const float dx1 = __fmul_rn((float)E.z, h), dx2 = __fmul_rn((float)E.w, h);
    f2 dx0s[2], du[2][3];
    float coef[2];
#pragma unroll
    for (int side = 0; side < 2; ++side) {
        if (!((SIDES >> side) & 1)) continue;
        const Own& O = side == 0 ? A : B;
        const float dx0 = __fmul_rn((float)(E.y - side), h);
        dx0s[side] = f2_make(dx0, dx0);
        for (int a = 0; a < 3; ++a) {
            const float v = split_diff(ujh[a], ujl[a], O.uh[a], O.ul[a]);
            du[side][a] = f2_make(v, v);
        }
        float c = O.c;
        if (BDRY) c *= 0.5f * (O.be + bej);
        if (SFAC) c *= 0.5f * (O.sf + sfj);
        coef[side] = c;
    }
    const f2 dx1s = f2_make(dx1, dx1), dx2s = f2_make(dx2, dx2);
    const float4* __restrict__ tab = d.sten_tab;
    const int nu = d.sten_nu;
    f2 F[2][3] = {{0ull, 0ull, 0ull}, {0ull, 0ull, 0ull}};
#pragma unroll
    for (int q = 0; q < 8; q += 4) {
        const float4 vx = __ldg(blk + (q >> 2) * N + j), vy = __ldg(blk + (2 + (q >> 2)) * N + j),
                     vz = __ldg(blk + (4 + (q >> 2)) * N + j);
#pragma unroll
        for (int kk = 0; kk < 2; ++kk) {
            const int k = (q >> 1) + kk;  // point pair (2k, 2k + 1)
            const f2 gx = kk ? f2_make(vx.z, vx.w) : f2_make(vx.x, vx.y);
            const f2 gy = kk ? f2_make(vy.z, vy.w) : f2_make(vy.x, vy.y);
            const f2 gz = kk ? f2_make(vz.z, vz.w) : f2_make(vz.x, vz.y);
            const f2 x1 = f2_add(dx1s, hy[k]), x2 = f2_add(dx2s, hz[k]);
#pragma unroll
            for (int side = 0; side < 2; ++side) {
                if (!((SIDES >> side) & 1)) continue;
                const float4 T = __ldg(tab + (side * nu + u) * 4 + k);  // K lo hi, 1/r^2 lo hi
                const f2 x0 = f2_add(dx0s[side], hx[k]);
                pt_force2<HASFAIL, SERIES>(x0, x1, x2, f2_make(T.x, T.y), f2_make(T.z, T.w),
                                           f2_add(du[side][0], gx), f2_add(du[side][1], gy),
                                           f2_add(du[side][2], gz), epsc[side], F[side], &wide);
            }
        }
    }
#pragma unroll
    for (int side = 0; side < 2; ++side) {
        if (!((SIDES >> side) & 1)) continue;
        float F6[6];
        f2_split(F[side][0], F6[0], F6[3]);
        f2_split(F[side][1], F6[1], F6[4]);
        f2_split(F[side][2], F6[2], F6[5]);
        float Fb[3];
        chains_sum(F6, Fb);
        kahan_add(side == 0 ? A : B, Fb, coef[side]);
    }
}

// Five blocks per SM (96 registers, 20 warps): the walk is latency-bound, and
// 4 blocks at 110 registers measured 5.00 against 4.70 ms per plate step
// (6 blocks at 80 registers: 4.71, with 104 bytes of spill).
// Two passes over the same tiles: EXACT = false evaluates every point with the
// series form alone (no branch between the point chains: 4.69 -> 3.9 ms of
// force per plate step); a tile in which any point left the series range
// stores nothing and is marked in sten_wide.  EXACT = true returns at once
// for unmarked tiles and evaluates the marked ones with the exact form where
// needed, then clears the mark.  Every point of every tile therefore takes
// the same operations as in the single-pass kernel.
template <bool HASFAIL, bool BDRY, bool SFAC, bool EXACT>
__global__ void __launch_bounds__(128, 5) k_force_f32c_sten(Dev d, PointPack<8> G, double dts) {
    if (EXACT) {
        const bool marked = d.sten_wide[blockIdx.x] != 0;
        __syncthreads();  // every thread has read the mark before it is cleared
        if (!marked) return;
        if (threadIdx.x == 0) d.sten_wide[blockIdx.x] = 0;
    }
    // the box of this tile: the last whose first tile is at most blockIdx.x
    int lo = 0, hi = d.sten_nbox - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&d.sten_box[mid].w) <= (int)blockIdx.x) lo = mid;
        else hi = mid - 1;
    }
    const int4 BX = __ldg(d.sten_box + lo);
    const longlong2 BB = __ldg(d.sten_boxb + lo);
    const int NX = BX.x, NY = BX.y, NZ = BX.z;
    const int64_t NXY = (int64_t)NX * NY;
    const int npx = (NX + 1) >> 1, TW = sten_tw(npx), BY = d.sten_by * (16 / TW), BZ = d.sten_bz;
    const int b = (int)blockIdx.x - BX.w;
    int px, y, z;
    if (sten_linear(npx, NY, NZ, TW, BY, BZ)) {  // 128 consecutive pairs of the box
        const int64_t lp = (int64_t)b * 128 + threadIdx.x;
        px = (int)(lp % npx);
        y = (int)((lp / npx) % NY);
        z = (int)(lp / ((int64_t)npx * NY));
    } else {
        const int nbx = (npx + TW - 1) / TW, nby = (NY + BY - 1) / BY;
        const int tx = threadIdx.x & (TW - 1), ty = threadIdx.x / TW;
        px = (b % nbx) * TW + tx;
        y = ((b / nbx) % nby) * BY + ty % BY;
        z = (b / (nbx * nby)) * BZ + ty / BY;
    }
    // threads past the box stay in the warp's walk with empty masks
    const bool valid = px < npx && y < NY && z < NZ;
    const int64_t NP = d.sten_np;
    const int64_t yz = valid ? y + (int64_t)NY * z : 0;
    const int64_t p = valid ? BB.y + px + (int64_t)npx * yz : 0;
    const int64_t ia = valid ? BB.x + 2 * px + (int64_t)NX * yz : 0;
    const bool hb = valid && 2 * px + 1 < NX;
    Own A, B;
    load_own<true, BDRY, SFAC, false>(d, ia, A);
    load_own<true, BDRY, SFAC, false>(d, hb ? ia + 1 : ia, B);
    const float epsc[2] = {HASFAIL ? eps_crit(A.e) : 0.f, HASFAIL ? eps_crit(B.e) : 0.f};
    const float h = (float)d.dx;
    f2 hx[4], hy[4], hz[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        hx[k] = f2_make(G.p[2 * k].hx, G.p[2 * k + 1].hx);
        hy[k] = f2_make(G.p[2 * k].hy, G.p[2 * k + 1].hy);
        hz[k] = f2_make(G.p[2 * k].hz, G.p[2 * k + 1].hz);
    }
    const int nw = d.sten_nw;
    int nba = 0, nbb = 0;
    bool wide = false;  // a point of this thread left the series range (series pass)
    for (int w = 0; w < nw; ++w) {
        const uint32_t ma = valid ? __ldg(d.sten_mask + (int64_t)w * NP + p) : 0u;
        const uint32_t mb = hb ? __ldg(d.sten_mask + (int64_t)(nw + w) * NP + p) : 0u;
        nba += __popc(ma);
        nbb += __popc(mb);
        uint32_t m = __reduce_or_sync(0xffffffffu, ma | mb);
        while (m) {
            const int bit = __ffs(m) - 1;
            m &= m - 1;
            const bool ha = ((ma >> bit) & 1u) != 0, hbit = ((mb >> bit) & 1u) != 0;
            const int u = 32 * w + bit;
            if (ha && hbit)
                sten_entry<HASFAIL, BDRY, SFAC, 3, !EXACT>(d, u, ia, NX, NXY, hx, hy, hz, epsc, h, A, B, wide);
            else if (ha)
                sten_entry<HASFAIL, BDRY, SFAC, 1, !EXACT>(d, u, ia, NX, NXY, hx, hy, hz, epsc, h, A, B, wide);
            else if (hbit)
                sten_entry<HASFAIL, BDRY, SFAC, 2, !EXACT>(d, u, ia, NX, NXY, hx, hy, hz, epsc, h, A, B, wide);
        }
    }
    if (!EXACT && __syncthreads_or(wide)) {  // left to the exact pass: nothing stored
        if (threadIdx.x == 0) d.sten_wide[blockIdx.x] = 1;
        return;
    }
    if (valid) store_own<false>(d, ia, A, nba, dts, d.vbuf);
    if (hb) store_own<false>(d, ia + 1, B, nbb, dts, d.vbuf);
}

// Setup of the stencil force's table: per U2 entry u, side (node A: offset
// o_u; node B = A + 1: o_u - e_x) and point pair k, K and 1/r^2 of the points
// 2k and 2k + 1 (pt_geo, from the same lattice-offset bond vector that bond4
// forms), laid out [side][u][k] as (K_2k, K_2k+1, 1/r2_2k, 1/r2_2k+1).
__global__ void k_sten_table(const int4* __restrict__ u2, int nu, PointPack<8> G, float h, float4* __restrict__ tab) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 8 * nu) return;
    const int k = t & 3, u = (t >> 2) % nu, side = t / (4 * nu);
    const int4 E = u2[u];
    const float dx0 = __fmul_rn((float)(E.y - side), h), dx1 = __fmul_rn((float)E.z, h),
                dx2 = __fmul_rn((float)E.w, h);
    float K[2], r2i[2];
    for (int l = 0; l < 2; ++l) {
        const PointF& P = G.p[2 * k + l];
        pt_geo(P, fadd(dx0, P.hx), fadd(dx1, P.hy), fadd(dx2, P.hz), K[l], r2i[l]);
    }
    tab[t] = make_float4(K[0], K[1], r2i[0], r2i[1]);
}

// Setup: the offsets (from the node) of every unbroken family entry, over
// [-R, R]^3.  err bit 1: a node id is not x + nx (y + ny z) of its lattice
// position; bit 2: an offset beyond R.
// the box of node i (boxes in node order)
__device__ __forceinline__ int sten_box_of_node(const Dev& d, int64_t i) {
    int lo = 0, hi = d.sten_nbox - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (d.sten_boxb[mid].x <= i) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__global__ void k_sten_offsets(Dev d, int R, int* __restrict__ bitmap, int* __restrict__ err) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= d.n) return;
    const int li = d.lat[i];
    const int xi = li & 2047, yi = (li >> 11) & 2047, zi = li >> 22;
    // node id = first + x + nx (y + ny z) of its position in its box
    const int bx = sten_box_of_node(d, i);
    const int4 BX = d.sten_box[bx];
    const int64_t f = d.sten_boxb[bx].x;
    const int l0 = d.lat[f];
    const int lx = xi - (l0 & 2047), ly = yi - ((l0 >> 11) & 2047), lz = zi - (l0 >> 22);
    if (lx < 0 || lx >= BX.x || ly < 0 || ly >= BX.y || lz < 0 || lz >= BX.z ||
        i != f + lx + (int64_t)BX.x * (ly + (int64_t)BX.y * lz))
        atomicOr(err, 1);
    const int W = 2 * R + 1;
    for (int64_t p = d.arow[i]; p < d.arow[i + 1]; ++p) {
        const int lj = d.lat[d.acol[p]];
        const int ox = (lj & 2047) - xi, oy = ((lj >> 11) & 2047) - yi, oz = (lj >> 22) - zi;
        if (abs(ox) > R || abs(oy) > R || abs(oz) > R) {
            atomicOr(err, 2);
            continue;
        }
        bitmap[(ox + R) + W * ((oy + R) + W * (oz + R))] = 1;  // same value from every writer
    }
}

// Setup: the two masks of every pair.  lut: U2 index of an offset from node
// A over [-R, R+1] x [-R, R] x [-R, R], or -1.  err bit 4: a family entry
// that is not in U2, not at A + its offset, or out of ascending order.
__global__ void k_sten_masks(Dev d, const int* __restrict__ lut, int R, uint32_t* __restrict__ mask,
                             int* __restrict__ err) {
    const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= d.sten_np) return;
    int bx = 0, hi = d.sten_nbox - 1;  // the box of pair p
    while (bx < hi) {
        const int mid = (bx + hi + 1) >> 1;
        if (d.sten_boxb[mid].y <= p) bx = mid;
        else hi = mid - 1;
    }
    const int4 BX = d.sten_box[bx];
    const int64_t lp = p - d.sten_boxb[bx].y;
    const int NX = BX.x, npx = (NX + 1) / 2;
    const int64_t NXY = (int64_t)NX * BX.y;
    const int px = (int)(lp % npx);
    const int64_t ia = d.sten_boxb[bx].x + 2 * px + (int64_t)NX * (lp / npx);
    const int la = d.lat[ia];
    const int xa = la & 2047, ya = (la >> 11) & 2047, za = la >> 22;
    const int WX = 2 * R + 2, W = 2 * R + 1;
    for (int side = 0; side < 2; ++side) {
        uint32_t m[16];
        for (int w = 0; w < 16; ++w) m[w] = 0u;
        if (side == 0 || 2 * px + 1 < NX) {
            const int64_t i = ia + side;
            int last = -1;
            for (int64_t e = d.arow[i]; e < d.arow[i + 1]; ++e) {
                const int64_t j = d.acol[e];
                const int lj = d.lat[j];
                const int ox = (lj & 2047) - xa, oy = ((lj >> 11) & 2047) - ya, oz = (lj >> 22) - za;
                int u = -1;
                if (ox >= -R && ox <= R + 1 && abs(oy) <= R && abs(oz) <= R)
                    u = lut[(ox + R) + WX * ((oy + R) + W * (oz + R))];
                if (u < 0 || u <= last ||
                    j != ia + d.sten_u2[u].y + (int64_t)NX * d.sten_u2[u].z + NXY * d.sten_u2[u].w) {
                    atomicOr(err, 4);
                    break;
                }
                m[u >> 5] |= 1u << (u & 31);
                last = u;
            }
        }
        for (int w = 0; w < d.sten_nw; ++w) mask[((int64_t)side * d.sten_nw + w) * d.sten_np + p] = m[w];
    }
}

// The same bond forces with the neighbour blocks of a lattice tile staged in
// shared memory.  A block owns a tile of tile_x x tile_y x tile_z lattice
// positions and copies the node blocks of the tile and of its halo (the
// family radius around it, clipped to the box) into shared memory, 144 bytes
// per node; every neighbour load of the force loop then reads shared memory,
// where a warp's 32 loads of different nodes take a few wavefronts instead
// of one L1 wavefront per node.  Thread t takes the x-adjacent pair of
// positions (x0 + 2 px, x0 + 2 px + 1) of the tile.  Same arithmetic per node
// as k_force_f32c_pair, so the same result bit for bit.
template <bool HASFAIL, bool BDRY, bool SFAC, bool MULTIMAT>
__global__ void __launch_bounds__(256, 1) k_force_f32c_tiled(Dev d, PointPack<8> G, double dts) {
    extern __shared__ float4 smem4[];
    float* smem = reinterpret_cast<float*>(smem4);
    const int TX = d.tile_x, TY = d.tile_y, TZ = d.tile_z, R = d.fam_radius;
    const int NX = d.lat_nx, NY = d.lat_ny, NZ = d.lat_nz;
    const int ntx = (NX + TX - 1) / TX, nty = (NY + TY - 1) / TY;
    const int b = blockIdx.x;
    const int x0 = (b % ntx) * TX, y0 = ((b / ntx) % nty) * TY, z0 = (b / (ntx * nty)) * TZ;
    const int lox = max(0, x0 - R), hix = min(NX, x0 + TX + R);
    const int loy = max(0, y0 - R), hiy = min(NY, y0 + TY + R);
    const int loz = max(0, z0 - R), hiz = min(NZ, z0 + TZ + R);
    const int LX = hix - lox, LY = hiy - loy, LZ = hiz - loz;
    const int L = LX * LY * LZ;
    for (int l = threadIdx.x; l < L; l += blockDim.x) {
        const int lx = l % LX, ly = (l / LX) % LY, lz = l / (LX * LY);
        const int id = d.pos2id[(lox + lx) + (int64_t)NX * ((loy + ly) + (int64_t)NY * (loz + lz))];
        if (id < 0) continue;
        const float4* src = reinterpret_cast<const float4*>(d.nblk + (int64_t)id * 32);
        float4* dst = reinterpret_cast<float4*>(smem + (int64_t)l * kTileStride);
#pragma unroll
        for (int q = 0; q < 8; ++q) dst[q] = __ldg(src + q);
    }
    __syncthreads();
    const int hx = TX / 2;
    const int t = threadIdx.x;
    if (t >= hx * TY * TZ) return;
    const int gx = x0 + 2 * (t % hx), gy = y0 + (t / hx) % TY, gz = z0 + t / (hx * TY);
    if (gx >= NX || gy >= NY || gz >= NZ) return;
    const int64_t row = (int64_t)NX * (gy + (int64_t)NY * gz);
    int64_t ia = d.pos2id[gx + row];
    int64_t ib = gx + 1 < NX ? d.pos2id[gx + 1 + row] : -1;
    if (ia < 0) {
        ia = ib;
        ib = -1;
    }
    if (ia < 0) return;
    const SmemTile T{smem, lox, loy, loz, LX, LY};
    force_nodes<HASFAIL, true, BDRY, SFAC, MULTIMAT, false, true>(d, G, dts, ia, ib, 0, 0.0, 0.0, T);
}

// the largest lattice offset along one axis over every active family entry
__global__ void k_family_radius(Dev d, int* out) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= d.n) return;
    const int li = d.lat[i];
    int r = 0;
    for (int64_t p = d.arow[i]; p < d.arow[i + 1]; ++p) {
        const int lj = d.lat[d.acol[p]];
        r = max(r, abs((lj & 2047) - (li & 2047)));
        r = max(r, abs(((lj >> 11) & 2047) - ((li >> 11) & 2047)));
        r = max(r, abs((lj >> 22) - (li >> 22)));
    }
    atomicMax(out, r);
}

// The same for any number of Gauss points (constants from shared memory).
template <bool SFAC>
__global__ void __launch_bounds__(128) k_force_f32c_any(Dev d, double dts) {
    __shared__ PointF sp[kMaxPoints];
    for (int g = threadIdx.x; g < d.npt; g += blockDim.x) {
        const GaussConst& Q = d.gc[g];
        sp[g] = PointF{Q.hgf[0], Q.hgf[1], Q.hgf[2], Q.Wf, Q.A, Q.B};
    }
    __syncthreads();
    const int64_t N = d.n;
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (tid >= N) return;
    const int64_t i = d.order[tid];
    const int npt = d.npt, bs = d.bs;
    const double* src = d.bc[i] >= 0 ? d.U : d.us;
    const double u0 = src[i], u1 = src[N + i], u2 = src[2 * N + i];
    const float uh0 = (float)u0, uh1 = (float)u1, uh2 = (float)u2;
    const float ul0 = (float)(u0 - (double)uh0), ul1 = (float)(u1 - (double)uh1), ul2 = (float)(u2 - (double)uh2);
    const float* si = d.sblk + 8 * i;
    const int mi = d.mat[i];
    const MatDev& Mi = d.mats[mi];
    float s0 = 0.f, s1 = 0.f, s2 = 0.f, k0 = 0.f, k1 = 0.f, k2 = 0.f;
    const int64_t pb = d.arow[i], pe = d.arow[i + 1];
    for (int64_t p = pb; p < pe; ++p) {
        const int64_t j = d.acol[p];
        const float* bj = d.nblk + j * bs;
        const float* sj = d.sblk + 8 * j;
        const float dx0 = (sj[0] - si[0]) + (sj[3] - si[3]);
        const float dx1 = (sj[1] - si[1]) + (sj[4] - si[4]);
        const float dx2 = (sj[2] - si[2]) + (sj[5] - si[5]);
        const float* uj = bj + 3 * npt;
        const float du0 = (uj[0] - uh0) + (uj[3] - ul0);
        const float du1 = (uj[1] - uh1) + (uj[4] - ul1);
        const float du2 = (uj[2] - uh2) + (uj[5] - ul2);
        const MatDev& Mj = d.mats[d.mat[j]];
        const float ecrit = (float)fmin(Mi.ecrit, Mj.ecrit);
        float coef = 0.5f * (si[6] + sj[6]) * (float)fmin(Mi.spring, Mj.spring);
        if (SFAC) coef *= 0.5f * (si[7] + sj[7]);
        float F0 = 0.f, F1 = 0.f, F2 = 0.f;
        for (int g = 0; g < npt; ++g) {
            const PointF& P = sp[g];
            const float x0 = dx0 + P.hx, x1 = dx1 + P.hy, x2 = dx2 + P.hz;
            const float e0 = du0 + bj[g], e1 = du1 + bj[npt + g], e2 = du2 + bj[2 * npt + g];
            const float y0 = x0 + e0, y1 = x1 + e1, y2 = x2 + e2;
            const float r2 = fmaf(x0, x0, fmaf(x1, x1, x2 * x2));
            const float dd = fmaf(e0, x0 + y0, fmaf(e1, x1 + y1, e2 * (x2 + y2)));
            const float p2 = r2 + dd;
            const float rinv = rsqrtf(r2), pinv = rsqrtf(p2);
            const float r = r2 * rinv;
            const float s = dd * rinv * __fdividef(1.0f, fmaf(p2, pinv, r));
            const float beta = __saturatef((P.A - r) * P.B);
            float fm = P.W * beta * s * pinv;
            if (dd > 0.f && s > ecrit) fm = 0.f;
            F0 = fmaf(fm, y0, F0);
            F1 = fmaf(fm, y1, F1);
            F2 = fmaf(fm, y2, F2);
        }
        F0 *= coef; F1 *= coef; F2 *= coef;
        float y = F0 - k0, t = s0 + y; k0 = (t - s0) - y; s0 = t;
        y = F1 - k1; t = s1 + y; k1 = (t - s1) - y; s1 = t;
        y = F2 - k2; t = s2 + y; k2 = (t - s2) - y; s2 = t;
    }
    const double rho = Mi.density, nb = (double)(pe - pb);
    d.vbuf[i] += ((double)s0 - (double)k0 + nb * (Mi.grav[0] * rho)) * dts / rho;
    d.vbuf[N + i] += ((double)s1 - (double)k1 + nb * (Mi.grav[1] * rho)) * dts / rho;
    d.vbuf[2 * N + i] += ((double)s2 - (double)k2 + nb * (Mi.grav[2] * rho)) * dts / rho;
}

// CCI in FP32 form: one point at node j, pdDataManager.cpp:1818-1866.  The
// effective displacement of every node (U for nodes with a boundary
// condition, us otherwise) is packed as hi/lo by k_pack_cci.
template <bool SFAC>
__global__ void __launch_bounds__(128) k_force_f32c_cci(Dev d, double dts) {
    const int64_t N = d.n;
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (tid >= N) return;
    const int64_t i = d.order[tid];
    const float* si = d.sblk + 8 * i;
    const float* ui = d.nblk + i * d.bs;
    const MatDev& Mi = d.mats[d.mat[i]];
    const float dl = (float)d.delta, h = (float)d.dx;
    const float outer = d.cci_mdf ? dl + 0.5f * h : dl;
    float s0 = 0.f, s1 = 0.f, s2 = 0.f, k0 = 0.f, k1 = 0.f, k2 = 0.f;
    const int64_t pb = d.arow[i], pe = d.arow[i + 1];
    for (int64_t p = pb; p < pe; ++p) {
        const int64_t j = d.acol[p];
        const float* sj = d.sblk + 8 * j;
        const float* uj = d.nblk + j * d.bs;
        const float x0 = (sj[0] - si[0]) + (sj[3] - si[3]);
        const float x1 = (sj[1] - si[1]) + (sj[4] - si[4]);
        const float x2 = (sj[2] - si[2]) + (sj[5] - si[5]);
        const float e0 = (uj[0] - ui[0]) + (uj[3] - ui[3]);
        const float e1 = (uj[1] - ui[1]) + (uj[4] - ui[4]);
        const float e2 = (uj[2] - ui[2]) + (uj[5] - ui[5]);
        const MatDev& Mj = d.mats[d.mat[j]];
        const float ecrit = (float)fmin(Mi.ecrit, Mj.ecrit);
        float coef = 0.5f * (si[6] + sj[6]) * (float)fmin(Mi.spring, Mj.spring) * (float)d.vol_cci;
        if (SFAC) coef *= 0.5f * (si[7] + sj[7]);
        const float y0 = x0 + e0, y1 = x1 + e1, y2 = x2 + e2;
        const float r2 = fmaf(x0, x0, fmaf(x1, x1, x2 * x2));
        const float dd = fmaf(e0, x0 + y0, fmaf(e1, x1 + y1, e2 * (x2 + y2)));
        const float p2 = r2 + dd;
        const float rinv = rsqrtf(r2), pinv = rsqrtf(p2);
        const float r = r2 * rinv;
        const float s = dd * rinv * __fdividef(1.0f, fmaf(p2, pinv, r));
        const float beta = (r > outer) ? 0.f : __saturatef((dl + 0.5f * h - r) / h);
        float fm = coef * beta * s * pinv;
        if (dd > 0.f && s > ecrit) fm = 0.f;
        const float F0 = fm * y0, F1 = fm * y1, F2 = fm * y2;
        float y = F0 - k0, t = s0 + y; k0 = (t - s0) - y; s0 = t;
        y = F1 - k1; t = s1 + y; k1 = (t - s1) - y; s1 = t;
        y = F2 - k2; t = s2 + y; k2 = (t - s2) - y; s2 = t;
    }
    const double rho = Mi.density, nb = (double)(pe - pb);
    d.vbuf[i] += ((double)s0 - (double)k0 + nb * (Mi.grav[0] * rho)) * dts / rho;
    d.vbuf[N + i] += ((double)s1 - (double)k1 + nb * (Mi.grav[1] * rho)) * dts / rho;
    d.vbuf[2 * N + i] += ((double)s2 - (double)k2 + nb * (Mi.grav[2] * rho)) * dts / rho;
}

__global__ void k_pack_cci(Dev d) {
    const int64_t N = d.n;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= N) return;
    const double* src = d.bc[i] >= 0 ? d.U : d.us;
    float* o = d.nblk + i * d.bs;
    for (int a = 0; a < 3; ++a) {
        const double u = src[a * N + i];
        const float hi = (float)u;
        o[a] = hi;
        o[3 + a] = (float)(u - (double)hi);
    }
}

// ----------------------------------------------------------------- gather

// Element e of node i's block: contiguous [N][bs], or chunk-major (float4
// chunk e / 4 of node i at nblk + 4 (chunk N + i)) for the lattice-stencil
// force, which reads chunk c of x-adjacent nodes side by side.
struct BlkOut {
    float* p;
    int64_t cs;  // 0: contiguous block; else the chunk stride 4 N
    __device__ __forceinline__ float& operator[](int e) const { return cs ? p[(e >> 2) * cs + (e & 3)] : p[e]; }
};
__device__ __forceinline__ BlkOut blk_out(const Dev& d, int64_t i) {
    return d.blk_cm ? BlkOut{d.nblk + 4 * i, 4 * d.n} : BlkOut{d.nblk + i * d.bs, 0};
}

// One thread per (node, group of up to four Gauss points): the Gauss-point
// displacement relative to the node, sum_k c_k (us_k - us_i) + (sum_k c_k - 1)
// us_i, accumulated in FP64 from FP32 coefficients (the MLS coefficients
// satisfy the partition of unity only to the accuracy the reference's
// ill-conditioned moment matrices allow, hence the second term).  Nodes with a
// boundary condition keep the reference's rules on the FP64 Gauss-point
// displacement (pdDataManager.cpp:2604-2703) and store its difference.
// SELL (sliced ELLPACK, 16 nodes per slice in the work order): contributor
// slot k of the 16 nodes of a slice is stored side by side, so a warp's index
// load reads 64 contiguous bytes and its coefficient load 512 (the CSR rows:
// one 32-byte sector in each of 16 rows).  Every thread still walks only its
// own node's contributors, in order: the same sums bit for bit.
// The part of a gather thread's work that needs no contributor: the node's
// trial displacement (u0, u1, u2) and its FP32 hi/lo split (group 0), and the
// whole job for nodes with a boundary condition or without MLS.  True when
// the thread is done.
template <bool PERSIST>
__device__ __forceinline__ bool gather_head(const Dev& d, const double* us, int64_t i, int grp, double t,
                                            const BlkOut& o, double& u0, double& u1, double& u2) {
    const int64_t N = d.n;
    const int npt = d.npt;
    const int g0 = 4 * grp, ng = min(4, npt - g0);
    u0 = ldm<PERSIST>(us + i);
    u1 = ldm<PERSIST>(us + N + i);
    u2 = ldm<PERSIST>(us + 2 * N + i);
    if (grp == 0) {
        const float h0 = (float)u0, h1 = (float)u1, h2 = (float)u2;
        o[3 * npt + 0] = h0;
        o[3 * npt + 1] = h1;
        o[3 * npt + 2] = h2;
        o[3 * npt + 3] = (float)(u0 - (double)h0);
        o[3 * npt + 4] = (float)(u1 - (double)h1);
        o[3 * npt + 5] = (float)(u2 - (double)h2);
    }
    const int b = d.bc[i];
    if (b >= 0) {
        const BcDev& B = d.bcs[b];
        const double fac = time_factor(B, t);
        for (int q = 0; q < ng; ++q) {
            const int g = g0 + q;
            double* ug = d.ug + (int64_t)(3 * g) * N + i;
            const GaussConst& G = d.gc[g];
            const double q0 = G.hg[0] + d.x[i], q1 = G.hg[1] + d.x[N + i], q2 = G.hg[2] + d.x[2 * N + i];
            for (int a = 0; a < 3; ++a) {
                if (B.dir[a] != 1) continue;
                if (B.type == PD_BC_DISPL) ug[a * N] = B.val[a] * fac;
                else if (B.type == PD_BC_DISPLGRAD)
                    ug[a * N] = (B.val[3 * a] * q0 + B.val[3 * a + 1] * q1 + B.val[3 * a + 2] * q2) * fac;
            }
            const double w0 = PERSIST ? __ldcg(ug) : ug[0];
            const double w1 = PERSIST ? __ldcg(ug + N) : ug[N];
            const double w2 = PERSIST ? __ldcg(ug + 2 * N) : ug[2 * N];
            o[g] = (float)(w0 - u0);
            o[npt + g] = (float)(w1 - u1);
            o[2 * npt + g] = (float)(w2 - u2);
        }
        return true;
    }
    if (!d.mls) {
        for (int q = 0; q < ng; ++q) o[g0 + q] = o[npt + g0 + q] = o[2 * npt + g0 + q] = 0.f;
        return true;
    }
    return false;
}

// PAT: contributor ids from the node's pattern (id offsets in an L1/L2-resident
// table) instead of its list; the index load then no longer waits on memory.
template <bool PERSIST, bool SELL = false, bool PAT = false>
__device__ __forceinline__ void gather_group(const Dev& d, const double* us, int64_t tid, double t) {
    const int64_t N = d.n;
    const int npt = d.npt, ngrp = (npt + 3) / 4;
    const int64_t i = d.order[tid / ngrp];
    const int grp = (int)(tid % ngrp);
    const int g0 = 4 * grp, ng = min(4, npt - g0);
    const BlkOut o = blk_out(d, i);
    double u0, u1, u2;
    if (gather_head<PERSIST>(d, us, i, grp, t, o, u0, u1, u2)) return;
    double a[4][3] = {};
    int64_t c0 = 0, nc = 0;
    const int32_t* po = nullptr;  // PAT: contributor k is i + po[k]
    if (PAT) {
        const int pid = __ldg(d.gpat_id + i);
        const int64_t q0 = __ldg(d.gpat_ptr + pid);
        nc = __ldg(d.gpat_ptr + pid + 1) - q0;
        po = d.gpat_off + q0;
        if (!SELL) c0 = d.cbptr[i];
    } else {
        c0 = d.cbptr[i];
        nc = d.cbptr[i + 1] - c0;
    }
    // contributor k: index cb[k * cs], coefficients cf[k * fs + q]
    const int32_t* cb = d.cbidx + c0;
    const float* cf = d.coeff32 + c0 * npt + g0;
    int64_t cs = 1, fs = npt;
    if (SELL) {
        const int64_t slot = tid / ngrp, sl = slot / kSell, l = slot % kSell, base = d.sell_off[sl];
        cb = d.sell_idx + base * kSell + l;
        cf = d.sell_coef + (base * kSell + l) * 8 + g0;
        cs = kSell;
        fs = kSell * 8;
    }
    const bool vec = (ng == 4) && ((npt & 3) == 0);
    int64_t k = 0;
    if (vec) {
        // four contributors per iteration: their index and displacement loads
        // are independent, which hides the index -> displacement latency
        for (; k + 4 <= nc; k += 4) {
            int m[4];
            float4 cv[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                m[u] = PAT ? (int)i + __ldg(po + k + u) : __ldg(cb + (k + u) * cs);
                cv[u] = ld4(cf + (k + u) * fs);
            }
            double dd[4][3];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                dd[u][0] = ldm<PERSIST>(us + m[u]) - u0;
                dd[u][1] = ldm<PERSIST>(us + N + m[u]) - u1;
                dd[u][2] = ldm<PERSIST>(us + 2 * N + m[u]) - u2;
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const float c[4] = {cv[u].x, cv[u].y, cv[u].z, cv[u].w};
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    a[q][0] = fma((double)c[q], dd[u][0], a[q][0]);
                    a[q][1] = fma((double)c[q], dd[u][1], a[q][1]);
                    a[q][2] = fma((double)c[q], dd[u][2], a[q][2]);
                }
            }
        }
    }
    for (; k < nc; ++k) {
        const int64_t m = PAT ? i + po[k] : cb[k * cs];
        const double d0 = ldm<PERSIST>(us + m) - u0, d1 = ldm<PERSIST>(us + N + m) - u1,
                     d2 = ldm<PERSIST>(us + 2 * N + m) - u2;
        float c[4];
        if (vec) {
            const float4 v = ld4(cf + k * fs);
            c[0] = v.x; c[1] = v.y; c[2] = v.z; c[3] = v.w;
        } else {
            for (int q = 0; q < 4; ++q) c[q] = q < ng ? cf[k * fs + q] : 0.f;
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            a[q][0] = fma((double)c[q], d0, a[q][0]);
            a[q][1] = fma((double)c[q], d1, a[q][1]);
            a[q][2] = fma((double)c[q], d2, a[q][2]);
        }
    }
    for (int q = 0; q < ng; ++q) {
        const double S = (double)d.csum[i * npt + g0 + q];
        o[g0 + q] = (float)fma(S, u0, a[q][0]);
        o[npt + g0 + q] = (float)fma(S, u1, a[q][1]);
        o[2 * npt + g0 + q] = (float)fma(S, u2, a[q][2]);
    }
}

template <bool SELL, bool PAT>
__global__ void __launch_bounds__(256) k_gather_f32c(Dev d, const double* __restrict__ us) {
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (tid >= d.n * ((d.npt + 3) / 4)) return;
    gather_group<false, SELL, PAT>(d, us, tid, *d.tdev);
}

// 16-byte copy global -> shared that the thread waits for later (L2 only:
// the coefficient stream is read once).
__device__ __forceinline__ void cp_async16(void* sdst, const void* gsrc) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gsrc) : "memory");
}
// the same with an L2 eviction policy (the coefficient stream is read once
// per gather: evict it first, so that the node blocks the force reads next
// stay in L2)
__device__ __forceinline__ uint64_t l2_evict_first() {
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
__device__ __forceinline__ void cp_async16_pol(void* sdst, const void* gsrc, uint64_t pol) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.cg.shared.global.L2::cache_hint [%0], [%1], 16, %2;" ::"r"(sa), "l"(gsrc), "l"(pol)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int NPEND>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(NPEND) : "memory");
}

// coefficient slots a thread keeps in flight: 64 KB of ring per block, two
// blocks per SM (12 slots in static shared memory: 1.84 ms per plate step;
// 16: 1.78; 24: 1.78)
constexpr int kRingSlots = 16;

// The SELL + pattern gather (2x2x2 points) with the coefficient stream run
// through a shared-memory ring: each thread copies its own 16 bytes of each
// contributor slot kRing slots ahead of the arithmetic (one commit group per
// slot), so a warp keeps about 8 KB of the stream in flight without holding
// it in registers; the contributor ids come from the node's pattern
// (L1-resident), and the contributors' trial displacements of the next group
// of four are loaded while the current group is summed.  A thread reads back only what it
// copied itself, after cp.async.wait_group, and refills a ring entry only
// after the values read from it have been used.  Same FMAs in the same
// contributor order as gather_group: the same result bit for bit.
template <int kRing>
__global__ void __launch_bounds__(256, 2) k_gather_f32c_ring(Dev d, const double* __restrict__ us) {
    extern __shared__ float4 ring_sm[];  // [8 warps][kRing][32 lanes]
    float4 (*ring)[kRing][32] = reinterpret_cast<float4 (*)[kRing][32]>(ring_sm);
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (tid >= d.n * 2) return;
    const int64_t N = d.n;
    const int64_t slot = tid >> 1;
    const int grp = (int)(tid & 1), g0 = 4 * grp;
    const int64_t i = d.order[slot];
    const BlkOut o = blk_out(d, i);
    double u0, u1, u2;
    if (gather_head<false>(d, us, i, grp, *d.tdev, o, u0, u1, u2)) return;
    const int pid = __ldg(d.gpat_id + i);
    const int64_t p0 = __ldg(d.gpat_ptr + pid);
    const int nc = (int)(__ldg(d.gpat_ptr + pid + 1) - p0);
    const int32_t* po = d.gpat_off + p0;
    const int64_t sl = slot / kSell, ln = slot % kSell, base = d.sell_off[sl];
    // contributor slot k of this thread: cf[32 k] (a slot is kSell nodes x 8 floats = 32 float4)
    const float4* cf = reinterpret_cast<const float4*>(d.sell_coef + (base * kSell + ln) * 8 + g0);
    float4* r = &ring[threadIdx.x >> 5][0][threadIdx.x & 31];  // ring entry e at r[32 e]
    const uint64_t pol = l2_evict_first();
#pragma unroll
    for (int k = 0; k < kRing; ++k) {
        if (k < nc) cp_async16_pol(r + 32 * k, cf + (int64_t)32 * k, pol);
        cp_async_commit();
    }
    // trial displacements of contributors k .. k+3, loaded one group ahead:
    // the two threads of a node (lanes 2s, 2s+1: same node, same pattern, the
    // same loop) each load two of the four (contributors k + 2v + grp) and
    // swap them with a pair-masked shuffle, so every displacement is loaded
    // once per node instead of once per thread
    const unsigned pair = 3u << (threadIdx.x & 30);
    double mine[2][3];
    auto load_group = [&](int k) {
#pragma unroll
        for (int v = 0; v < 2; ++v) {
            const int u = 2 * v + grp;
            const int m = (int)i + (k + u < nc ? __ldg(po + k + u) : 0);
            mine[v][0] = __ldg(us + m);
            mine[v][1] = __ldg(us + N + m);
            mine[v][2] = __ldg(us + 2 * N + m);
        }
    };
    load_group(0);
    double a[4][3] = {};
    int e = 0;  // ring entry of contributor k
    for (int k = 0; k < nc; k += 4) {
        double dd[4][3];
#pragma unroll
        for (int v = 0; v < 2; ++v) {
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const double other = __shfl_xor_sync(pair, mine[v][c], 1);
                dd[2 * v][c] = grp ? other : mine[v][c];
                dd[2 * v + 1][c] = grp ? mine[v][c] : other;
            }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            dd[u][0] -= u0;
            dd[u][1] -= u1;
            dd[u][2] -= u2;
        }
        if (k + 4 < nc) load_group(k + 4);
        cp_async_wait<kRing - 4>();  // slots k .. k+3 have landed
        float4 cv[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int eu = e + u < kRing ? e + u : e + u - kRing;
            cv[u] = k + u < nc ? r[32 * eu] : make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (k + u >= nc) break;
            const float c[4] = {cv[u].x, cv[u].y, cv[u].z, cv[u].w};
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                a[q][0] = fma((double)c[q], dd[u][0], a[q][0]);
                a[q][1] = fma((double)c[q], dd[u][1], a[q][1]);
                a[q][2] = fma((double)c[q], dd[u][2], a[q][2]);
            }
        }
        // refill the four entries just used with slots k + kRing .. k + kRing + 3
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int eu = e + u < kRing ? e + u : e + u - kRing;
            const int kk = k + kRing + u;
            if (kk < nc) cp_async16_pol(r + 32 * eu, cf + (int64_t)32 * kk, pol);
            cp_async_commit();
        }
        e = e + 4 < kRing ? e + 4 : e + 4 - kRing;
    }
    cp_async_wait<0>();
    for (int q = 0; q < 4; ++q) {
        const double S = (double)d.csum[i * 8 + g0 + q];
        o[g0 + q] = (float)fma(S, u0, a[q][0]);
        o[8 + g0 + q] = (float)fma(S, u1, a[q][1]);
        o[16 + g0 + q] = (float)fma(S, u2, a[q][2]);
    }
}

// FP64 Gauss-point displacements from the node blocks the FP32 gather wrote:
// us_j (hi + lo) plus the point's FP32 offset (the adjoint's stage tape of
// the FP32-compensated form).
__global__ void k_blocks_to_ug(Dev d, double* __restrict__ ug) {
    const int64_t N = d.n;
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= N) return;
    const int npt = d.npt;
    const BlkOut o = blk_out(d, j);
    for (int a = 0; a < 3; ++a) {
        const double u = (double)o[3 * npt + a] + (double)o[3 * npt + 3 + a];
        for (int g = 0; g < npt; ++g) ug[(int64_t)(3 * g + a) * N + j] = u + (double)o[a * npt + g];
    }
}

// SELL layout: the widest contributor list of every slice, then the copy
__global__ void k_sell_width(Dev d, int64_t* __restrict__ width, int64_t S) {
    const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (s >= S) return;
    int64_t w = 0;
    for (int l = 0; l < kSell; ++l) {
        const int64_t slot = s * kSell + l;
        if (slot >= d.n) break;
        const int64_t i = d.order[slot];
        w = max(w, d.cbptr[i + 1] - d.cbptr[i]);
    }
    width[s] = w;
}

__global__ void k_sell_fill(Dev d, const int64_t* __restrict__ off, int32_t* __restrict__ sidx,
                            float* __restrict__ scoef) {
    const int64_t slot = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (slot >= d.n) return;
    const int64_t i = d.order[slot], sl = slot / kSell, l = slot % kSell, base = off[sl];
    const int64_t c0 = d.cbptr[i], nc = d.cbptr[i + 1] - c0;
    for (int64_t k = 0; k < nc; ++k) {
        sidx[(base + k) * kSell + l] = d.cbidx[c0 + k];
        const float* src = d.coeff32 + (c0 + k) * 8;
        float* dst = scoef + ((base + k) * kSell + l) * 8;
        for (int g = 0; g < 8; ++g) dst[g] = src[g];
    }
}

// The same gather with one thread per (node, Gauss point): a third of the
// registers, so more warps and more contributor loads in flight; the eight
// threads of a node read its coefficients of one contributor as 32
// contiguous bytes and share the contributor's index and displacement loads.
__global__ void __launch_bounds__(256) k_gather_f32c_pt(Dev d, const double* __restrict__ us) {
    const int64_t N = d.n;
    const int npt = d.npt;
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (tid >= N * npt) return;
    const int64_t i = d.order[tid / npt];
    const int g = (int)(tid % npt);
    const double t = *d.tdev;
    const double u0 = __ldg(us + i), u1 = __ldg(us + N + i), u2 = __ldg(us + 2 * N + i);
    const BlkOut o = blk_out(d, i);
    if (g == 0) {
        const float h0 = (float)u0, h1 = (float)u1, h2 = (float)u2;
        o[3 * npt + 0] = h0;
        o[3 * npt + 1] = h1;
        o[3 * npt + 2] = h2;
        o[3 * npt + 3] = (float)(u0 - (double)h0);
        o[3 * npt + 4] = (float)(u1 - (double)h1);
        o[3 * npt + 5] = (float)(u2 - (double)h2);
    }
    const int b = d.bc[i];
    if (b >= 0) {
        const BcDev& B = d.bcs[b];
        const double fac = time_factor(B, t);
        double* ug = d.ug + (int64_t)(3 * g) * N + i;
        const GaussConst& G = d.gc[g];
        const double q0 = G.hg[0] + d.x[i], q1 = G.hg[1] + d.x[N + i], q2 = G.hg[2] + d.x[2 * N + i];
        for (int a = 0; a < 3; ++a) {
            if (B.dir[a] != 1) continue;
            if (B.type == PD_BC_DISPL) ug[a * N] = B.val[a] * fac;
            else if (B.type == PD_BC_DISPLGRAD)
                ug[a * N] = (B.val[3 * a] * q0 + B.val[3 * a + 1] * q1 + B.val[3 * a + 2] * q2) * fac;
        }
        o[g] = (float)(ug[0] - u0);
        o[npt + g] = (float)(ug[N] - u1);
        o[2 * npt + g] = (float)(ug[2 * N] - u2);
        return;
    }
    if (!d.mls) {
        o[g] = o[npt + g] = o[2 * npt + g] = 0.f;
        return;
    }
    const int64_t c0 = d.cbptr[i], nc = d.cbptr[i + 1] - c0;
    const int32_t* cb = d.cbidx + c0;
    const float* cf = d.coeff32 + c0 * npt + g;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    int64_t k = 0;
    for (; k + 4 <= nc; k += 4) {
        int m[4];
        float c[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            m[u] = __ldg(cb + k + u);
            c[u] = __ldg(cf + (k + u) * npt);
        }
        double v[4][3];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            v[u][0] = __ldg(us + m[u]) - u0;
            v[u][1] = __ldg(us + N + m[u]) - u1;
            v[u][2] = __ldg(us + 2 * N + m[u]) - u2;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            a0 = fma((double)c[u], v[u][0], a0);
            a1 = fma((double)c[u], v[u][1], a1);
            a2 = fma((double)c[u], v[u][2], a2);
        }
    }
    for (; k < nc; ++k) {
        const int64_t m = cb[k];
        const double cc = (double)cf[k * npt];
        a0 = fma(cc, us[m] - u0, a0);
        a1 = fma(cc, us[N + m] - u1, a1);
        a2 = fma(cc, us[2 * N + m] - u2, a2);
    }
    const double S = (double)d.csum[i * npt + g];
    o[g] = (float)fma(S, u0, a0);
    o[npt + g] = (float)fma(S, u1, a1);
    o[2 * npt + g] = (float)fma(S, u2, a2);
}

// ------------------------------------------------------------ persistent

// Grid barrier for one cooperative launch (all blocks co-resident).  The
// arrival counter only grows: barrier k of the launch is passed once it
// reaches (k+1) * gridDim.x.  The wait is bounded: after W.ns nanoseconds
// without completion the block sets the error word and every block leaves at
// its next barrier; the host reads the word and reports PD_ERR_TIMEOUT.
// W.stall (tests of that path only): block 0 does not arrive at the first
// barrier, so every wait there runs out.

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ bool grid_barrier(PersistCtl* ctl, unsigned& passed, const PersistWait& W) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        const unsigned target = (passed + 1) * gridDim.x;
        __threadfence();
        if (!(W.stall && blockIdx.x == 0 && passed == 0)) atomicAdd(&ctl->arrive, 1u);
        const unsigned long long t0 = global_ns();
        for (;;) {
            const unsigned a = *((volatile unsigned*)&ctl->arrive);
            if (a >= target) break;
            if (*((volatile int*)&ctl->error) != 0) { ok = 0; break; }
            if (global_ns() - t0 > W.ns) {
                atomicExch(&ctl->error, 1);
                ok = 0;
                break;
            }
            __nanosleep(100);
        }
        __threadfence();
    }
    __syncthreads();
    ++passed;
    return ok != 0;
}

// One work-queue phase: blocks take chunks of `chunk` items from a counter
// of their own (one counter per phase of the launch, zeroed before it).
template <typename F>
__device__ __forceinline__ void run_queue(unsigned* counter, int64_t nitems, unsigned chunk, F&& work) {
    __shared__ unsigned long long base_s;
    for (;;) {
        if (threadIdx.x == 0) base_s = (unsigned long long)atomicAdd(counter, chunk);
        __syncthreads();
        const int64_t base = (int64_t)base_s;
        __syncthreads();
        if (base >= nitems) break;
        const int64_t end = base + chunk < nitems ? base + chunk : nitems;
        for (int64_t it = base + threadIdx.x; it < end; it += blockDim.x) work(it);
    }
}

// nsteps RK4 steps of the FP32-compensated FGI form (2x2x2 points) in one
// launch.  Per stage two phases separated by grid barriers: (a) the bond
// forces of node pairs fused with the stage epilogue of both nodes, (b) the
// MLS gather of the trial displacement (of U after stage 4).  Same arithmetic
// as the separate launches of one graph-captured step, so the same result bit
// for bit.  The time advances as k_advance_time advances it.
template <bool HASFAIL, bool LAT, bool BDRY, bool SFAC, bool MULTIMAT>
__global__ void __launch_bounds__(128, 4) k_persist_f32c(Dev d, PointPack<8> G, double dt, int nsteps,
                                                         PersistCtl* ctl, unsigned force_chunk,
                                                         unsigned gather_chunk, PersistWait W) {
    const int64_t N = d.n;
    const int64_t npairs = (N + 1) / 2;
    const int64_t ngather = N * ((d.npt + 3) / 4);
    unsigned passed = 0;
    // every block reads the start time before the first barrier; block 0
    // writes the end time after the last one
    double t = __ldcg(d.tdev);
    const double dtHalf = 0.5 * dt;
    for (int step = 0; step < nsteps; ++step) {
        t = t + dt;
        for (int stage = 1; stage <= 4; ++stage) {
            const double dts = stage <= 2 ? dtHalf : dt;
            unsigned* q = ctl->next + 8 * (int64_t)step + 2 * (stage - 1);
            run_queue(q, npairs, force_chunk, [&](int64_t it) {
                force_pair<HASFAIL, LAT, BDRY, SFAC, MULTIMAT, true>(d, G, dts, 2 * it, stage, dt, t);
            });
            if (!grid_barrier(ctl, passed, W)) return;
            const double* src = stage < 4 ? d.us : d.U;
            run_queue(q + 1, ngather, gather_chunk, [&](int64_t it) { gather_group<true>(d, src, it, t); });
            if (!grid_barrier(ctl, passed, W)) return;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *d.tdev = t;
}

template <int NPT>
PointPack<NPT> pack_points(const Dev& d, const GaussConst* host_gc) {
    PointPack<NPT> P;
    for (int g = 0; g < NPT; ++g)
        P.p[g] = PointF{host_gc[g].hgf[0], host_gc[g].hgf[1], host_gc[g].hgf[2], host_gc[g].Wf, host_gc[g].A,
                        host_gc[g].B};
    return P;
}

}  // namespace

size_t tiled_smem_bytes(const Dev& d) {
    const int R = d.fam_radius;
    const int64_t lx = std::min(d.lat_nx, d.tile_x + 2 * R), ly = std::min(d.lat_ny, d.tile_y + 2 * R),
                  lz = std::min(d.lat_nz, d.tile_z + 2 * R);
    return (size_t)(lx * ly * lz) * kTileStride * sizeof(float);
}

int prepare_tiled_force(size_t smem) {
    const void* fns[] = {(const void*)k_force_f32c_tiled<true, true, true, true>,
                         (const void*)k_force_f32c_tiled<false, true, true, false>,
                         (const void*)k_force_f32c_tiled<false, true, false, false>,
                         (const void*)k_force_f32c_tiled<false, false, true, false>,
                         (const void*)k_force_f32c_tiled<false, false, false, false>};
    for (const void* f : fns)
        if (cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
            return PD_ERR_CUDA;
    return PD_OK;
}

void launch_family_radius(const Dev& d, int* out, cudaStream_t s) {
    cudaMemsetAsync(out, 0, sizeof(int), s);
    if (d.n > 0 && d.lat) k_family_radius<<<blocks_for(d.n, 256), 256, 0, s>>>(d, out);
}

void launch_blocks_to_ug(const Dev& d, double* ug, cudaStream_t s) {
    if (d.n) k_blocks_to_ug<<<blocks_for(d.n, 256), 256, 0, s>>>(d, ug);
}

void launch_force_f32c(const Dev& d, double dts, cudaStream_t s) {
    if (d.n == 0) return;
    const unsigned nb = blocks_for(d.n, 128);
    if (d.cci) {
        k_pack_cci<<<blocks_for(d.n, 256), 256, 0, s>>>(d);
        if (d.sfac) k_force_f32c_cci<true><<<nb, 128, 0, s>>>(d, dts);
        else k_force_f32c_cci<false><<<nb, 128, 0, s>>>(d, dts);
        return;
    }
    if (d.blk_cm && d.sten_mask && d.npt == 8 && d.gc_host) {
        // the gather stores chunk-major blocks: only this kernel reads them
        const unsigned nbk = (unsigned)d.sten_ntiles;
        const bool bd = d.bdry_on != 0, sf = d.sfac != nullptr;
        const PointPack<8> P = pack_points<8>(d, d.gc_host);
#define PD_STEN(HF, BD, SF)                                              \
    do {                                                                 \
        k_force_f32c_sten<HF, BD, SF, false><<<nbk, 128, 0, s>>>(d, P, dts); \
        k_force_f32c_sten<HF, BD, SF, true><<<nbk, 128, 0, s>>>(d, P, dts);  \
    } while (0)
        if (d.hasfail) {
            if (bd) { if (sf) PD_STEN(true, true, true); else PD_STEN(true, true, false); }
            else { if (sf) PD_STEN(true, false, true); else PD_STEN(true, false, false); }
        } else {
            if (bd) { if (sf) PD_STEN(false, true, true); else PD_STEN(false, true, false); }
            else { if (sf) PD_STEN(false, false, true); else PD_STEN(false, false, false); }
        }
#undef PD_STEN
        return;
    }
    if (d.npt == 8 && d.gc_host && d.tile_x > 0 && d.lat && d.pos2id) {
        const PointPack<8> P = pack_points<8>(d, d.gc_host);
        const int nt = ((d.lat_nx + d.tile_x - 1) / d.tile_x) * ((d.lat_ny + d.tile_y - 1) / d.tile_y) *
                       ((d.lat_nz + d.tile_z - 1) / d.tile_z);
        const int bs = d.tile_x / 2 * d.tile_y * d.tile_z;
        const size_t sh = tiled_smem_bytes(d);
        const bool bd = d.bdry_on != 0, sf = d.sfac != nullptr;
        if (d.hasfail || d.multimat) k_force_f32c_tiled<true, true, true, true><<<nt, bs, sh, s>>>(d, P, dts);
        else if (bd) {
            if (sf) k_force_f32c_tiled<false, true, true, false><<<nt, bs, sh, s>>>(d, P, dts);
            else k_force_f32c_tiled<false, true, false, false><<<nt, bs, sh, s>>>(d, P, dts);
        } else {
            if (sf) k_force_f32c_tiled<false, false, true, false><<<nt, bs, sh, s>>>(d, P, dts);
            else k_force_f32c_tiled<false, false, false, false><<<nt, bs, sh, s>>>(d, P, dts);
        }
        return;
    }
    if (d.npt == 8 && d.gc_host && d.force_quad && d.lat && !d.hasfail && !d.multimat) {
        const PointPack<8> P = pack_points<8>(d, d.gc_host);
        const unsigned nq = blocks_for((d.n + 3) / 4, 128);
        const bool bd = d.bdry_on != 0, sf = d.sfac != nullptr;
        if (bd) {
            if (sf) k_force_f32c_quad<true, true><<<nq, 128, 0, s>>>(d, P, dts);
            else k_force_f32c_quad<true, false><<<nq, 128, 0, s>>>(d, P, dts);
        } else {
            if (sf) k_force_f32c_quad<false, true><<<nq, 128, 0, s>>>(d, P, dts);
            else k_force_f32c_quad<false, false><<<nq, 128, 0, s>>>(d, P, dts);
        }
        return;
    }
    if (d.npt == 8 && d.gc_host) {
        const PointPack<8> P = pack_points<8>(d, d.gc_host);
        const unsigned np = blocks_for((d.n + 1) / 2, 128);
        const bool lat = d.lat != nullptr, bd = d.bdry_on != 0, sf = d.sfac != nullptr;
#define PD_F32(HF, LT, BD, SF, MM) k_force_f32c_pair<HF, LT, BD, SF, MM><<<np, 128, 0, s>>>(d, P, dts)
        if (d.hasfail || d.multimat) {
            PD_F32(true, false, true, true, true);
        } else if (lat) {
            if (bd) { if (sf) PD_F32(false, true, true, true, false); else PD_F32(false, true, true, false, false); }
            else { if (sf) PD_F32(false, true, false, true, false); else PD_F32(false, true, false, false, false); }
        } else {
            if (bd) { if (sf) PD_F32(false, false, true, true, false); else PD_F32(false, false, true, false, false); }
            else { if (sf) PD_F32(false, false, false, true, false); else PD_F32(false, false, false, false, false); }
        }
#undef PD_F32
        return;
    }
    if (d.sfac) k_force_f32c_any<true><<<nb, 128, 0, s>>>(d, dts);
    else k_force_f32c_any<false><<<nb, 128, 0, s>>>(d, dts);
}

// The persistent kernel's variant for the problem, and how many of its
// blocks fit on the device at once (a cooperative launch needs all resident).
namespace {
using PersistFn = void (*)(Dev, PointPack<8>, double, int, PersistCtl*, unsigned, unsigned, PersistWait);
PersistFn persist_variant(const Dev& d) {
    const bool lat = d.lat != nullptr, bd = d.bdry_on != 0, sf = d.sfac != nullptr;
    if (d.hasfail || d.multimat) return k_persist_f32c<true, false, true, true, true>;
    if (lat) {
        if (bd) return sf ? k_persist_f32c<false, true, true, true, false> : k_persist_f32c<false, true, true, false, false>;
        return sf ? k_persist_f32c<false, true, false, true, false> : k_persist_f32c<false, true, false, false, false>;
    }
    if (bd) return sf ? k_persist_f32c<false, false, true, true, false> : k_persist_f32c<false, false, true, false, false>;
    return sf ? k_persist_f32c<false, false, false, true, false> : k_persist_f32c<false, false, false, false, false>;
}
}  // namespace

int persist_max_blocks(const Dev& d, int* per_sm, int* sms) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return PD_ERR_CUDA;
    if (cudaDeviceGetAttribute(sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return PD_ERR_CUDA;
    int coop = 0;
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    if (!coop) return PD_ERR_CUDA;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, persist_variant(d), 128, 0) != cudaSuccess)
        return PD_ERR_CUDA;
    return PD_OK;
}

cudaError_t launch_persist_f32c(const Dev& d, double dt, int nsteps, PersistCtl* ctl, int blocks,
                                unsigned force_chunk, unsigned gather_chunk, PersistWait W, cudaStream_t s) {
    const PointPack<8> P = pack_points<8>(d, d.gc_host);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)blocks);
    cfg.blockDim = dim3(128);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    // its gather and force phases use the contiguous node blocks
    Dev t = d;
    t.blk_cm = 0;
    return cudaLaunchKernelEx(&cfg, persist_variant(t), t, P, dt, nsteps, ctl, force_chunk, gather_chunk, W);
}

void launch_gather_f32c(const Dev& d, const double* us, cudaStream_t s) {
    if (d.cci || d.n == 0) return;
    if (d.gather_per_point) {
        k_gather_f32c_pt<<<blocks_for(d.n * d.npt, 256), 256, 0, s>>>(d, us);
        return;
    }
    const int ngrp = (d.npt + 3) / 4;
    const unsigned nb = blocks_for(d.n * ngrp, 256);
    const bool sell = d.sell_on && d.sell_idx && d.mls && d.npt == 8, pat = d.gpat_id && d.mls;
    if (sell && pat && d.npt == 8) {
        static bool attr = false;  // once per process: the ring needs more than the 48 KB default
        const size_t sh = (size_t)8 * kRingSlots * 32 * sizeof(float4);
        if (!attr) {
            cudaFuncSetAttribute(k_gather_f32c_ring<kRingSlots>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
            attr = true;
        }
        k_gather_f32c_ring<kRingSlots><<<nb, 256, sh, s>>>(d, us);
    } else if (sell) {
        if (pat) k_gather_f32c<true, true><<<nb, 256, 0, s>>>(d, us);
        else k_gather_f32c<true, false><<<nb, 256, 0, s>>>(d, us);
    } else {
        if (pat) k_gather_f32c<false, true><<<nb, 256, 0, s>>>(d, us);
        else k_gather_f32c<false, false><<<nb, 256, 0, s>>>(d, us);
    }
}

int64_t sell_slices(const Dev& d) { return (d.n + kSell - 1) / kSell; }

void launch_sten_offsets(const Dev& d, int R, int* bitmap, int* err, cudaStream_t s) {
    if (d.n) k_sten_offsets<<<blocks_for(d.n, 256), 256, 0, s>>>(d, R, bitmap, err);
}

void launch_sten_masks(const Dev& d, const int* lut, int R, uint32_t* mask, int* err, cudaStream_t s) {
    if (d.sten_np) k_sten_masks<<<blocks_for(d.sten_np, 128), 128, 0, s>>>(d, lut, R, mask, err);
}


int launch_sten_table(const Dev& d, float4* tab, cudaStream_t s) {
    if (d.sten_nu <= 0 || !d.gc_host) return PD_ERR_ARG;
    const PointPack<8> P = pack_points<8>(d, d.gc_host);
    k_sten_table<<<blocks_for(8 * d.sten_nu, 128), 128, 0, s>>>(d.sten_u2, d.sten_nu, P, (float)d.dx, tab);
    return cudaGetLastError() == cudaSuccess ? PD_OK : PD_ERR_CUDA;
}


void launch_sell_width(const Dev& d, int64_t* width, cudaStream_t s) {
    const int64_t S = sell_slices(d);
    if (S) k_sell_width<<<blocks_for(S, 256), 256, 0, s>>>(d, width, S);
}

void launch_sell_fill(const Dev& d, const int64_t* off, int32_t* sidx, float* scoef, cudaStream_t s) {
    if (d.n) k_sell_fill<<<blocks_for(d.n, 128), 128, 0, s>>>(d, off, sidx, scoef);
}

void launch_pack_cci_f32c(const Dev& d, cudaStream_t s) {
    if (!d.cci || d.n == 0) return;
    k_pack_cci<<<blocks_for(d.n, 256), 256, 0, s>>>(d);
}

}  // namespace pd
