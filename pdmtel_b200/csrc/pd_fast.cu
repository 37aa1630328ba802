// The static operator (FP64 and FP32 matvec, right-hand side), the CG pieces,
// scans and reductions.
#include <cstdio>
#include <type_traits>

#include "pd_internal.cuh"

namespace pd {

namespace {

inline unsigned blocks_for(int64_t n, int bs) { return (unsigned)((n + bs - 1) / bs); }

__device__ __forceinline__ double time_factor(const BcDev& b, double t) {
    if (b.type == PD_BC_VELOC) return (t <= b.end_time) ? 1.0 : 0.0;
    if (b.load_type == 1.0) return (t <= b.end_time) ? t / b.end_time : 1.0;
    return 1.0;
}

// -------------------------------------------------------- static operator

__device__ __forceinline__ void prescribed(const Dev& d, int64_t i, double t, bool* pre, double* val) {
    pre[0] = pre[1] = pre[2] = false;
    val[0] = val[1] = val[2] = 0.0;
    const int b = d.bc[i];
    if (b < 0) return;
    const BcDev& B = d.bcs[b];
    if (B.type != PD_BC_DISPL && B.type != PD_BC_VELOC) return;
    for (int a = 0; a < 3; ++a)
        if (B.dir[a] == 1) {
            pre[a] = true;
            val[a] = (B.type == PD_BC_DISPL) ? B.val[a] : B.val[a] * t;
        }
}

// y = K x on free rows (prescribed columns masked), y = x on prescribed rows.
// One thread per node over its unbroken family; pdSolve.cpp:195-527.
template <bool SFAC>
__global__ void k_static_apply_f64(Dev d, double t, const double* __restrict__ x, double* __restrict__ y) {
    const int64_t N = d.n;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= N) return;
    bool pi[3];
    double pv[3];
    prescribed(d, i, t, pi, pv);
    const double X0 = d.x[i], X1 = d.x[N + i], X2 = d.x[2 * N + i];
    const double xi0 = pi[0] ? 0.0 : x[i], xi1 = pi[1] ? 0.0 : x[N + i], xi2 = pi[2] ? 0.0 : x[2 * N + i];
    const double ci = d.mats[d.mat[i]].spring;
    const double sfi = SFAC ? d.sfac[i] : 0.0;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    for (int64_t p = d.arow[i]; p < d.arow[i + 1]; ++p) {
        const int64_t j = d.acol[p];
        bool pj[3];
        double qv[3];
        prescribed(d, j, t, pj, qv);
        const double e0 = d.x[j] - X0, e1 = d.x[N + j] - X1, e2 = d.x[2 * N + j] - X2;
        const double r2 = e0 * e0 + e1 * e1 + e2 * e2;
        const double r = sqrt(r2);
        const double cj = d.mats[d.mat[j]].spring;
        double c = (cj < ci) ? cj : ci;
        if (SFAC) c = c * (0.5 * (sfi + d.sfac[j]));
        const double w = c * d.vol / (r2 * r);
        const double d0 = xi0 - (pj[0] ? 0.0 : x[j]);
        const double d1 = xi1 - (pj[1] ? 0.0 : x[N + j]);
        const double d2 = xi2 - (pj[2] ? 0.0 : x[2 * N + j]);
        const double pr = w * (e0 * d0 + e1 * d1 + e2 * d2);
        a0 += pr * e0;
        a1 += pr * e1;
        a2 += pr * e2;
    }
    y[i] = pi[0] ? x[i] : a0;
    y[N + i] = pi[1] ? x[N + i] : a1;
    y[2 * N + i] = pi[2] ? x[2 * N + i] : a2;
}

// The same operator with FP32 arithmetic on FP64 vectors: the per-bond
// difference x_i - x_j is formed in FP64 and rounded once, the bond term is
// FP32, the node sum FP64.  The matvec of the mixed-precision CG.
template <bool SFAC>
__global__ void k_static_apply_f32x(Dev d, double t, const double* __restrict__ x, double* __restrict__ y) {
    const int64_t N = d.n;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= N) return;
    bool pi[3];
    double pv[3];
    prescribed(d, i, t, pi, pv);
    const double X0 = d.x[i], X1 = d.x[N + i], X2 = d.x[2 * N + i];
    const double xi0 = pi[0] ? 0.0 : x[i], xi1 = pi[1] ? 0.0 : x[N + i], xi2 = pi[2] ? 0.0 : x[2 * N + i];
    const double ci = d.mats[d.mat[i]].spring;
    const double sfi = SFAC ? d.sfac[i] : 0.0;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    for (int64_t p = d.arow[i]; p < d.arow[i + 1]; ++p) {
        const int64_t j = d.acol[p];
        bool pj[3];
        double qv[3];
        prescribed(d, j, t, pj, qv);
        const float e0 = (float)(d.x[j] - X0), e1 = (float)(d.x[N + j] - X1), e2 = (float)(d.x[2 * N + j] - X2);
        const double cj = d.mats[d.mat[j]].spring;
        double c = (cj < ci) ? cj : ci;
        if (SFAC) c = c * (0.5 * (sfi + d.sfac[j]));
        const float rinv = rsqrtf(fmaf(e0, e0, fmaf(e1, e1, e2 * e2)));
        const float w = (float)(c * d.vol) * rinv * rinv * rinv;
        const float d0 = (float)(xi0 - (pj[0] ? 0.0 : x[j]));
        const float d1 = (float)(xi1 - (pj[1] ? 0.0 : x[N + j]));
        const float d2 = (float)(xi2 - (pj[2] ? 0.0 : x[2 * N + j]));
        const float pr = w * fmaf(e0, d0, fmaf(e1, d1, e2 * d2));
        a0 += (double)(pr * e0);
        a1 += (double)(pr * e1);
        a2 += (double)(pr * e2);
    }
    y[i] = pi[0] ? x[i] : a0;
    y[N + i] = pi[1] ? x[N + i] : a1;
    y[2 * N + i] = pi[2] ? x[2 * N + i] : a2;
}

// prescribed directions of every node as bits 0..2 (the static operator's
// masks do not depend on the time)
__global__ void k_static_pmask(Dev d, uint8_t* __restrict__ pm) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= d.n) return;
    bool pr[3];
    double v[3];
    prescribed(d, i, 0.0, pr, v);
    pm[i] = (uint8_t)((pr[0] ? 1 : 0) | (pr[1] ? 2 : 0) | (pr[2] ? 4 : 0));
}

// The operator on a complete box lattice whose families are the horizon
// stencil clipped to the box: the neighbour of slot k is i + off[k].w when
// the shifted lattice position stays in the box; the bond geometry and
// c V / r^3 come from the stencil table (one material).  No family list and
// no coordinates are read.  Threads take nodes in lattice order, so for one
// stencil slot a warp reads 32 consecutive neighbours; nodes at least the
// stencil radius inside the box skip the box test.  The input arrives
// masked (prescribed components zeroed, k_static_mask): FP64, or rounded to
// FP32 for the FP32 operator.  (An FP32 hi/lo split of the input, for
// FP64-accurate neighbour differences, loads as many bytes as FP64 and did
// not lower the CG iteration count on the 128^3 cube: 700 against 650.)
template <typename T>
__global__ void k_static_mask(const uint8_t* __restrict__ pmask, int64_t N, const double* __restrict__ x,
                              T* __restrict__ xm) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= N) return;
    const unsigned m = pmask[i];
    for (int a = 0; a < 3; ++a) {
        const double v = (m & (1u << a)) ? 0.0 : x[a * N + i];
        xm[a * N + i] = (T)v;
    }
}

// FP64: bond terms and sums in FP64.  FP32: bond terms in FP32 from an FP32
// copy of the table, summed in FP32 over runs of 16 stencil slots and then
// added to the FP64 node sum (conversions run on the scarce XU pipe).
template <typename T, bool SFAC, bool CHECK>
__device__ __forceinline__ void stencil_sum(const Dev& d, const StencilDev& S, const double4* sgeo,
                                            const float4* sgeof, const int4* soff, int64_t i, int ix, int iy,
                                            int iz, const T* __restrict__ xm, double sfi, double& a0, double& a1,
                                            double& a2) {
    const int64_t N = d.n;
    a0 = a1 = a2 = 0.0;
    if (sizeof(T) == 4) {
        const float* __restrict__ h0 = reinterpret_cast<const float*>(xm);
        const float* __restrict__ h1 = h0 + N;
        const float* __restrict__ h2 = h0 + 2 * N;
        const float hi0 = h0[i], hi1 = h1[i], hi2 = h2[i];
        for (int k0 = 0; k0 < S.ns; k0 += 16) {
            float s0 = 0.f, s1 = 0.f, s2 = 0.f;
            const int ke = min(k0 + 16, S.ns);
#pragma unroll 4
            for (int k = k0; k < ke; ++k) {
                const int4 o = soff[k];
                if (CHECK && ((unsigned)(ix + o.x) >= (unsigned)S.nx || (unsigned)(iy + o.y) >= (unsigned)S.ny ||
                              (unsigned)(iz + o.z) >= (unsigned)S.nz))
                    continue;
                const int64_t j = i + o.w;
                const float4 g = sgeof[k];
                float w = g.w;
                if (SFAC) w *= (float)(0.5 * (sfi + d.sfac[j]));
                const float d0 = hi0 - h0[j], d1 = hi1 - h1[j], d2 = hi2 - h2[j];
                const float pr = w * fmaf(g.x, d0, fmaf(g.y, d1, g.z * d2));
                s0 = fmaf(pr, g.x, s0);
                s1 = fmaf(pr, g.y, s1);
                s2 = fmaf(pr, g.z, s2);
            }
            a0 += (double)s0;
            a1 += (double)s1;
            a2 += (double)s2;
        }
    } else {
        const double* __restrict__ x0p = reinterpret_cast<const double*>(xm);
        const double* __restrict__ x1p = x0p + N;
        const double* __restrict__ x2p = x0p + 2 * N;
        const double xi0 = x0p[i], xi1 = x1p[i], xi2 = x2p[i];
#pragma unroll 4
        for (int k = 0; k < S.ns; ++k) {
            const int4 o = soff[k];
            if (CHECK && ((unsigned)(ix + o.x) >= (unsigned)S.nx || (unsigned)(iy + o.y) >= (unsigned)S.ny ||
                          (unsigned)(iz + o.z) >= (unsigned)S.nz))
                continue;
            const int64_t j = i + o.w;
            const double4 g = sgeo[k];
            double w = g.w;
            if (SFAC) w = w * (0.5 * (sfi + d.sfac[j]));
            const double d0 = xi0 - x0p[j], d1 = xi1 - x1p[j], d2 = xi2 - x2p[j];
            const double pr = w * (g.x * d0 + g.y * d1 + g.z * d2);
            a0 += pr * g.x;
            a1 += pr * g.y;
            a2 += pr * g.z;
        }
    }
}

template <typename T, bool SFAC>
__global__ void __launch_bounds__(256) k_static_stencil(Dev d, StencilDev S, const double* __restrict__ x,
                                                        const T* __restrict__ xm, double* __restrict__ y) {
    extern __shared__ double4 sgeo[];
    float4* sgeof = reinterpret_cast<float4*>(sgeo + S.ns);
    int4* soff = reinterpret_cast<int4*>(sgeof + S.ns);
    for (int k = threadIdx.x; k < S.ns; k += blockDim.x) {
        const double4 g = S.geo[k];
        sgeo[k] = g;
        sgeof[k] = make_float4((float)g.x, (float)g.y, (float)g.z, (float)g.w);
        soff[k] = S.off[k];
    }
    __syncthreads();
    const int64_t N = d.n;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int ix = (int)(i % S.nx), iy = (int)((i / S.nx) % S.ny), iz = (int)(i / ((int64_t)S.nx * S.ny));
    const unsigned mi = S.pmask[i];
    const double sfi = SFAC ? d.sfac[i] : 0.0;
    double a0, a1, a2;
    const int R = S.radius;
    const bool inner = ix >= R && ix < S.nx - R && iy >= R && iy < S.ny - R && iz >= R && iz < S.nz - R;
    if (inner) stencil_sum<T, SFAC, false>(d, S, sgeo, sgeof, soff, i, ix, iy, iz, xm, sfi, a0, a1, a2);
    else stencil_sum<T, SFAC, true>(d, S, sgeo, sgeof, soff, i, ix, iy, iz, xm, sfi, a0, a1, a2);
    y[i] = (mi & 1) ? x[i] : a0;
    y[N + i] = (mi & 2) ? x[N + i] : a1;
    y[2 * N + i] = (mi & 4) ? x[2 * N + i] : a2;
}

// Block-Jacobi preconditioner of the static operator: per node the inverse
// of its 3x3 diagonal block sum_j c V_j xi xi^T / r^3 over the unbroken
// family (the coefficients of pdSolve::AssembleEquation), with prescribed
// directions as identity rows and columns; stored symmetric [6][N] (xx yy zz
// xy xz yz).  A singular block (a node without bonds) keeps the identity.
template <bool SFAC>
__global__ void k_static_bjacobi(Dev d, double* __restrict__ minv) {
    const int64_t N = d.n;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= N) return;
    bool pi[3];
    double pv[3];
    prescribed(d, i, 0.0, pi, pv);
    const double X0 = d.x[i], X1 = d.x[N + i], X2 = d.x[2 * N + i];
    const double ci = d.mats[d.mat[i]].spring;
    const double sfi = SFAC ? d.sfac[i] : 0.0;
    double D[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int64_t p = d.arow[i]; p < d.arow[i + 1]; ++p) {
        const int64_t j = d.acol[p];
        const double e[3] = {d.x[j] - X0, d.x[N + j] - X1, d.x[2 * N + j] - X2};
        const double r2 = e[0] * e[0] + e[1] * e[1] + e[2] * e[2];
        const double r = sqrt(r2);
        const double cj = d.mats[d.mat[j]].spring;
        double c = (cj < ci) ? cj : ci;
        if (SFAC) c = c * (0.5 * (sfi + d.sfac[j]));
        const double w = c * d.vol / (r2 * r);
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) D[a][b] += w * e[a] * e[b];
    }
    for (int a = 0; a < 3; ++a)
        if (pi[a])
            for (int b = 0; b < 3; ++b) D[a][b] = D[b][a] = (a == b) ? 1.0 : 0.0;
    // inverse by cofactors (D symmetric)
    const double c00 = D[1][1] * D[2][2] - D[1][2] * D[2][1];
    const double c01 = D[1][2] * D[2][0] - D[1][0] * D[2][2];
    const double c02 = D[1][0] * D[2][1] - D[1][1] * D[2][0];
    const double det = D[0][0] * c00 + D[0][1] * c01 + D[0][2] * c02;
    double m[6] = {1.0, 1.0, 1.0, 0.0, 0.0, 0.0};
    if (det > 0.0 && isfinite(det)) {
        const double id = 1.0 / det;
        m[0] = c00 * id;
        m[1] = (D[0][0] * D[2][2] - D[0][2] * D[2][0]) * id;
        m[2] = (D[0][0] * D[1][1] - D[0][1] * D[1][0]) * id;
        m[3] = c01 * id;
        m[4] = c02 * id;
        m[5] = (D[0][2] * D[1][0] - D[0][0] * D[1][2]) * id;
    }
    for (int k = 0; k < 6; ++k) minv[k * N + i] = m[k];
}

// z = M^-1 r with the blocks of k_static_bjacobi
__global__ void k_bj_apply(const double* __restrict__ minv, const double* __restrict__ r, double* __restrict__ z,
                           int64_t N) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        const double r0 = r[i], r1 = r[N + i], r2 = r[2 * N + i];
        const double m0 = minv[i], m1 = minv[N + i], m2 = minv[2 * N + i];
        const double m3 = minv[3 * N + i], m4 = minv[4 * N + i], m5 = minv[5 * N + i];
        z[i] = m0 * r0 + m3 * r1 + m4 * r2;
        z[N + i] = m3 * r0 + m1 * r1 + m5 * r2;
        z[2 * N + i] = m4 * r0 + m5 * r1 + m2 * r2;
    }
}

// The same operator blocked along z: a thread owns R consecutive nodes of a
// z column, (ix, iy, iz0 .. iz0 + R - 1), and walks the stencil by (ox, oy)
// columns; every neighbour value of a column window z in [iz0 - rz, iz0 + R
// - 1 + rz] is loaded once and serves the up to 2 rz + 1 bonds of the R nodes
// that reach it, so a node needs (R + 2 rz) / R loads per column instead of
// one per bond.  The oz window is padded with zero weights where an offset is
// not in the stencil.  Sums per node in column order; FP32 bond terms are
// added in FP32 over four columns, then to the FP64 sum.
template <typename T, bool SFAC, int RZ, int R>
__global__ void __launch_bounds__(128) k_static_zcol(Dev d, StencilDev S, const double* __restrict__ x,
                                                     const T* __restrict__ xm, double* __restrict__ y) {
    constexpr int W = 2 * RZ + 1;
    using G = typename std::conditional<sizeof(T) == 4, float4, double4>::type;
    extern __shared__ double4 zsm[];
    G* geo = reinterpret_cast<G*>(zsm);
    int4* cols = reinterpret_cast<int4*>(geo + S.ncol * W);
    for (int k = threadIdx.x; k < S.ncol * W; k += blockDim.x) {
        const double4 g = S.colgeo[k];
        geo[k] = G{(T)g.x, (T)g.y, (T)g.z, (T)g.w};
    }
    for (int k = threadIdx.x; k < S.ncol; k += blockDim.x) cols[k] = S.col[k];
    __syncthreads();
    const int64_t N = d.n, nxy = (int64_t)S.nx * S.ny;
    const int ix = blockIdx.x * 32 + (threadIdx.x & 31);
    const int iy = blockIdx.y * 4 + (threadIdx.x >> 5);
    const int iz0 = blockIdx.z * R;
    const bool in_xy = ix < S.nx && iy < S.ny;
    const int64_t i0 = ix + (int64_t)S.nx * iy + nxy * iz0;
    T xi[R][3];
    double sfi[R];
#pragma unroll
    for (int m = 0; m < R; ++m) {
        const bool v = in_xy && iz0 + m < S.nz;
        for (int a = 0; a < 3; ++a) xi[m][a] = v ? xm[a * N + i0 + m * nxy] : (T)0;
        sfi[m] = (SFAC && v) ? d.sfac[i0 + m * nxy] : 0.0;
    }
    double acc[R][3];
    T part[R][3];
#pragma unroll
    for (int m = 0; m < R; ++m)
        for (int a = 0; a < 3; ++a) acc[m][a] = 0.0, part[m][a] = (T)0;
    for (int c = 0; c < S.ncol; ++c) {
        const int4 C = cols[c];
        const bool cv = in_xy && (unsigned)(ix + C.x) < (unsigned)S.nx && (unsigned)(iy + C.y) < (unsigned)S.ny;
        G g[W];
#pragma unroll
        for (int q = 0; q < W; ++q) g[q] = geo[c * W + q];
#pragma unroll
        for (int zz = -RZ; zz < R + RZ; ++zz) {
            const int jz = iz0 + zz;
            if (!cv || jz < 0 || jz >= S.nz) continue;
            const int64_t j = i0 + C.z + nxy * zz;
            const T xj0 = xm[j], xj1 = xm[N + j], xj2 = xm[2 * N + j];
            const double sfj = SFAC ? d.sfac[j] : 0.0;
#pragma unroll
            for (int m = 0; m < R; ++m) {
                const int oz = zz - m;
                if (oz < -RZ || oz > RZ) continue;
                const G& q = g[oz + RZ];
                T w = q.w;
                if (SFAC) w = w * (T)(0.5 * (sfi[m] + sfj));
                const T d0 = xi[m][0] - xj0, d1 = xi[m][1] - xj1, d2 = xi[m][2] - xj2;
                const T pr = w * (q.x * d0 + q.y * d1 + q.z * d2);
                part[m][0] += pr * q.x;
                part[m][1] += pr * q.y;
                part[m][2] += pr * q.z;
            }
        }
        if (sizeof(T) == 8 || (c & 3) == 3 || c + 1 == S.ncol) {
#pragma unroll
            for (int m = 0; m < R; ++m)
                for (int a = 0; a < 3; ++a) {
                    acc[m][a] += (double)part[m][a];
                    part[m][a] = (T)0;
                }
        }
    }
#pragma unroll
    for (int m = 0; m < R; ++m) {
        if (!in_xy || iz0 + m >= S.nz) continue;
        const int64_t i = i0 + m * nxy;
        const unsigned mi = S.pmask[i];
        y[i] = (mi & 1) ? x[i] : acc[m][0];
        y[N + i] = (mi & 2) ? x[N + i] : acc[m][1];
        y[2 * N + i] = (mi & 4) ? x[2 * N + i] : acc[m][2];
    }
}

// The FP64 operator in the split form K x = D_i x_i - sum_o W_o x_(i+o), with
// W_o = w_o xi_o xi_o^T and D_i = sum of W_o over the offsets that stay in the
// box (k_static_ndiag; the same block for every node at least the stencil
// reach inside the box).  A column (ox, oy) of the stencil contributes
// -sum_oz w (a_j + ez pz_j) (ex, ey, ez) with a_j = ex px_j + ey py_j formed
// once per loaded neighbour, so a bond costs three FMAs: s = a + ez pz,
// T += w s, TZ += (w ez) s, and the column adds (ex T, ey T, TZ) to the node.
// Columns come sorted by their half-height h (the offsets of a column are oz
// in [-h, h]; missing ones have w = 0), so every class runs with its own
// unrolled window.  FP64 only: in FP32 the cancellation of D_i x_i against
// the neighbour sum is not a rounding of the input and slows CG down.
//
// A block owns a tile of 32 x 4 x R nodes (a thread: R consecutive nodes of a
// z column) and first stages the tile and its stencil halo, (32 + 2 rx) x
// (4 + 2 ry) x (R + 2 rz) nodes of the masked input (k_static_mask), in
// shared memory with asynchronous copies that are all in flight before the
// block waits once; positions outside the box are zero-filled, so a
// neighbour there adds nothing and the bond loop has no box test.  Every
// neighbour value is read from L2 once per block instead of once per column
// window of every thread.  (Reading the neighbours straight from global
// memory ran at a 54% L1 hit rate, latency-bound on the misses: 511 us per
// 128^3 matvec.)
__device__ __forceinline__ void cp_async8z(double* sdst, const double* gsrc, bool valid) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(sa), "l"(gsrc), "r"(valid ? 8 : 0)
                 : "memory");
}
// The tile has a halo of RH nodes on every side (RH = the stencil's largest
// offset component), so every shared-memory offset below is a compile-time
// constant.
template <int R, int RH>
struct NdTile {
    static constexpr int LX = 32 + 2 * RH, LY = 4 + 2 * RH, LZ = R + 2 * RH;
    static constexpr int SS = LX * LY, CS = SS * LZ;
};

template <int H, int R, int RH>
__device__ __forceinline__ void nd_column(const double* __restrict__ b, const double* ez,
                                          const double2* __restrict__ tap, double ex, double ey,
                                          double (&acc)[R][3]) {
    using L = NdTile<R, RH>;
    constexpr int W = 2 * H + 1;
    double w[W], wz[W];
#pragma unroll
    for (int q = 0; q < W; ++q) {
        const double2 t = tap[4 - H + q];
        w[q] = t.x;
        wz[q] = t.y;
    }
    double T[R], TZ[R];
#pragma unroll
    for (int m = 0; m < R; ++m) T[m] = TZ[m] = 0.0;
#pragma unroll
    for (int zz = -H; zz < R + H; ++zz) {
        const double px = b[zz * L::SS], py = b[L::CS + zz * L::SS], pz = b[2 * L::CS + zz * L::SS];
        const double a = fma(ey, py, ex * px);
#pragma unroll
        for (int m = 0; m < R; ++m) {
            const int oz = zz - m;
            if (oz < -H || oz > H) continue;
            const double s = fma(ez[oz + H], pz, a);
            T[m] = fma(w[oz + H], s, T[m]);
            TZ[m] = fma(wz[oz + H], s, TZ[m]);
        }
    }
#pragma unroll
    for (int m = 0; m < R; ++m) {
        acc[m][0] = fma(-ex, T[m], acc[m][0]);
        acc[m][1] = fma(-ey, T[m], acc[m][1]);
        acc[m][2] -= TZ[m];
    }
}

template <int H, int R, int RH>
__device__ __forceinline__ void nd_class(const NdTab& tb, int c0, int c1, int g, const double* own, double sp,
                                         double (&acc)[R][3]) {
    if (H > RH) return;
    double ez[2 * H + 1];
#pragma unroll
    for (int q = 0; q <= 2 * H; ++q) ez[q] = (q - H) * sp;
    for (int c = c0 + g; c < c1; c += 2) {
        const int4 C = tb.col[c];
        nd_column<H, R, RH>(own + C.y * NdTile<R, RH>::LX + C.x, ez, tb.tap + c * 9, C.x * sp, C.y * sp, acc);
    }
}

// the halo of the tile: the stencil's largest offset component (0 when it
// is beyond 4: the difference form runs instead)
inline int nd_halo(const StencilDev& S) {
    const int h = S.nrx > S.nry ? (S.nrx > S.rz ? S.nrx : S.rz) : (S.nry > S.rz ? S.nry : S.rz);
    return h <= 4 ? h : 0;
}

// shared memory of k_static_nd: the staged tile [3][LZ][LY][LX]
inline size_t nd_smem(const StencilDev& S, int R) {
    const size_t h = nd_halo(S);
    const size_t LX = 32 + 2 * h, LY = 4 + 2 * h, LZ = R + 2 * h;
    return 3 * LX * LY * LZ * sizeof(double);
}

// 256 threads: two groups of 128 take the even and the odd columns of every
// class for the same nodes (twice the warps per staged tile), and the second
// group hands its sums to the first through shared memory.
template <int R, int RH>
__global__ void __launch_bounds__(256) k_static_nd(Dev d, StencilDev S, const __grid_constant__ NdTab tb,
                                                   const double* __restrict__ x, const double* __restrict__ xm,
                                                   double* __restrict__ y) {
    using L = NdTile<R, RH>;
    extern __shared__ double2 ndsm[];
    double* P = reinterpret_cast<double*>(ndsm);
    const int64_t N = d.n, nxy = (int64_t)S.nx * S.ny;
    const int x0 = blockIdx.x * 32, y0 = blockIdx.y * 4, z0 = blockIdx.z * R;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // stage the tile and its halo: one row of LX nodes per warp at a time
    for (int row = warp; row < L::LY * L::LZ; row += 8) {
        const int ly = row % L::LY, lz = row / L::LY;
        const int gy = y0 - RH + ly, gz = z0 - RH + lz;
        const bool rv = gy >= 0 && gy < S.ny && gz >= 0 && gz < S.nz;
        const int64_t jr = (int64_t)gy * S.nx + nxy * gz;
#pragma unroll
        for (int lx0 = 0; lx0 < L::LX; lx0 += 32) {
            const int lx = lx0 + lane;
            if (lx >= L::LX) break;
            const int gx = x0 - RH + lx;
            const bool v = rv && gx >= 0 && gx < S.nx;
            const int64_t j = v ? jr + gx : 0;  // zero-filled copies read nothing
            const int k = row * L::LX + lx;
            cp_async8z(P + k, xm + j, v);
            cp_async8z(P + L::CS + k, xm + N + j, v);
            cp_async8z(P + 2 * L::CS + k, xm + 2 * N + j, v);
        }
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncthreads();
    const int g = warp >> 2;  // column group
    const int tx = lane, ty = warp & 3;
    const int ix = x0 + tx, iy = y0 + ty;
    // this thread's first node in the tile
    const double* own = P + RH * L::SS + (ty + RH) * L::LX + (tx + RH);
    double acc[R][3];
#pragma unroll
    for (int m = 0; m < R; ++m) acc[m][0] = acc[m][1] = acc[m][2] = 0.0;
    const double sp = S.sp;
    nd_class<0, R, RH>(tb, S.ndcls[0], S.ndcls[1], g, own, sp, acc);
    nd_class<1, R, RH>(tb, S.ndcls[1], S.ndcls[2], g, own, sp, acc);
    nd_class<2, R, RH>(tb, S.ndcls[2], S.ndcls[3], g, own, sp, acc);
    nd_class<3, R, RH>(tb, S.ndcls[3], S.ndcls[4], g, own, sp, acc);
    nd_class<4, R, RH>(tb, S.ndcls[4], S.ndcls[5], g, own, sp, acc);
    // the own values the first group still needs, then the second group's
    // sums through the (no longer read) tile
    double u[R][3];
#pragma unroll
    for (int m = 0; m < R; ++m) {
        u[m][0] = own[m * L::SS];
        u[m][1] = own[L::CS + m * L::SS];
        u[m][2] = own[2 * L::CS + m * L::SS];
    }
    __syncthreads();
    double* xch = P + (threadIdx.x & 127);
    if (g == 1) {
#pragma unroll
        for (int m = 0; m < R; ++m)
            for (int a = 0; a < 3; ++a) xch[(3 * m + a) * 128] = acc[m][a];
    }
    __syncthreads();
    if (g == 1 || ix >= S.nx || iy >= S.ny) return;
#pragma unroll
    for (int m = 0; m < R; ++m)
        for (int a = 0; a < 3; ++a) acc[m][a] += xch[(3 * m + a) * 128];
    const bool xy_inner = S.ndin && ix >= S.nrx && ix < S.nx - S.nrx && iy >= S.nry && iy < S.ny - S.nry;
    const int64_t i0 = ix + (int64_t)S.nx * iy + nxy * z0;
#pragma unroll
    for (int m = 0; m < R; ++m) {
        const int iz = z0 + m;
        if (iz >= S.nz) continue;
        const int64_t i = i0 + m * nxy;
        const bool inner = xy_inner && iz >= S.rz && iz < S.nz - S.rz;
        double D[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) D[k] = inner ? S.ndint[k] : S.ndiag[k * N + i];
        const double u0 = u[m][0], u1 = u[m][1], u2 = u[m][2];
        const double y0v = fma(D[0], u0, fma(D[3], u1, fma(D[4], u2, acc[m][0])));
        const double y1v = fma(D[3], u0, fma(D[1], u1, fma(D[5], u2, acc[m][1])));
        const double y2v = fma(D[4], u0, fma(D[5], u1, fma(D[2], u2, acc[m][2])));
        const unsigned mi = S.pmask[i];
        y[i] = (mi & 1) ? x[i] : y0v;
        y[N + i] = (mi & 2) ? x[N + i] : y1v;
        y[2 * N + i] = (mi & 4) ? x[2 * N + i] : y2v;
    }
}

// D_i = sum of w xi xi^T over the stencil offsets that stay in the box, from
// the column tables k_static_nd reads: blocks (00, 11, 22, 01, 02, 12).
__global__ void k_static_ndiag(StencilDev S, int64_t N, double* __restrict__ D) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int ix = (int)(i % S.nx), iy = (int)((i / S.nx) % S.ny), iz = (int)(i / ((int64_t)S.nx * S.ny));
    double a[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int c = 0; c < S.ndcol; ++c) {
        const int4 C = S.ndc[c];
        if ((unsigned)(ix + C.x) >= (unsigned)S.nx || (unsigned)(iy + C.y) >= (unsigned)S.ny) continue;
        const double ex = C.x * S.sp, ey = C.y * S.sp;
        for (int oz = -C.w; oz <= C.w; ++oz) {
            if ((unsigned)(iz + oz) >= (unsigned)S.nz) continue;
            const double w = S.ndtap[c * 9 + 4 + oz].x, ez = oz * S.sp;
            a[0] += w * ex * ex;
            a[1] += w * ey * ey;
            a[2] += w * ez * ez;
            a[3] += w * ex * ey;
            a[4] += w * ex * ez;
            a[5] += w * ey * ez;
        }
    }
    for (int k = 0; k < 6; ++k) D[k * N + i] = a[k];
}

template <int R, int RH>
void launch_nd_h(const Dev& d, const StencilDev& S, const double* x, const double* xm, double* y, cudaStream_t s) {
    const dim3 grid((unsigned)((S.nx + 31) / 32), (unsigned)((S.ny + 3) / 4), (unsigned)((S.nz + R - 1) / R));
    static bool attr = false;  // once per process: the tile needs more than the 48 KB default
    if (!attr) {
        cudaFuncSetAttribute(k_static_nd<R, RH>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        attr = true;
    }
    k_static_nd<R, RH><<<grid, 256, nd_smem(S, R), s>>>(d, S, *S.ndhost, x, xm, y);
}

template <int R>
void launch_nd(const Dev& d, const StencilDev& S, const double* x, const double* xm, double* y, cudaStream_t s) {
    switch (nd_halo(S)) {
        case 1: launch_nd_h<R, 1>(d, S, x, xm, y, s); break;
        case 2: launch_nd_h<R, 2>(d, S, x, xm, y, s); break;
        case 3: launch_nd_h<R, 3>(d, S, x, xm, y, s); break;
        default: launch_nd_h<R, 4>(d, S, x, xm, y, s); break;
    }
}

template <typename T, bool SFAC, int R>
void launch_zcol(const Dev& d, const StencilDev& S, const double* x, const T* xm, double* y, cudaStream_t s) {
    const dim3 grid((unsigned)((S.nx + 31) / 32), (unsigned)((S.ny + 3) / 4), (unsigned)((S.nz + R - 1) / R));
    const size_t sh = (size_t)S.ncol * (2 * S.rz + 1) * (sizeof(T) == 4 ? sizeof(float4) : sizeof(double4)) +
                      (size_t)S.ncol * sizeof(int4);
    switch (S.rz) {
        case 1: k_static_zcol<T, SFAC, 1, R><<<grid, 128, sh, s>>>(d, S, x, xm, y); break;
        case 2: k_static_zcol<T, SFAC, 2, R><<<grid, 128, sh, s>>>(d, S, x, xm, y); break;
        case 3: k_static_zcol<T, SFAC, 3, R><<<grid, 128, sh, s>>>(d, S, x, xm, y); break;
        default: k_static_zcol<T, SFAC, 4, R><<<grid, 128, sh, s>>>(d, S, x, xm, y); break;
    }
}

// b = prescribed values on prescribed rows; on free rows the moved prescribed
// columns (pdSolve.cpp:296-363 sign pattern) plus the traction load.
template <bool SFAC>
__global__ void k_static_rhs(Dev d, double t, double* __restrict__ out) {
    const int64_t N = d.n;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= N) return;
    bool pi[3];
    double pv[3];
    prescribed(d, i, t, pi, pv);
    const double X0 = d.x[i], X1 = d.x[N + i], X2 = d.x[2 * N + i];
    const double ci = d.mats[d.mat[i]].spring;
    const double sfi = SFAC ? d.sfac[i] : 0.0;
    const double m0 = pi[0] ? pv[0] : 0.0, m1 = pi[1] ? pv[1] : 0.0, m2 = pi[2] ? pv[2] : 0.0;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    for (int64_t p = d.arow[i]; p < d.arow[i + 1]; ++p) {
        const int64_t j = d.acol[p];
        bool pj[3];
        double qv[3];
        prescribed(d, j, t, pj, qv);
        const double e0 = d.x[j] - X0, e1 = d.x[N + j] - X1, e2 = d.x[2 * N + j] - X2;
        const double r2 = e0 * e0 + e1 * e1 + e2 * e2;
        const double r = sqrt(r2);
        const double cj = d.mats[d.mat[j]].spring;
        double c = (cj < ci) ? cj : ci;
        if (SFAC) c = c * (0.5 * (sfi + d.sfac[j]));
        const double w = c * d.vol / (r2 * r);
        // -K_ii(prescribed cols) ubar_i + K_ij-part: +c xi xi^T ubar_j
        const double d0 = (pj[0] ? qv[0] : 0.0) - m0;
        const double d1 = (pj[1] ? qv[1] : 0.0) - m1;
        const double d2 = (pj[2] ? qv[2] : 0.0) - m2;
        const double pr = w * (e0 * d0 + e1 * d1 + e2 * d2);
        a0 += pr * e0;
        a1 += pr * e1;
        a2 += pr * e2;
    }
    double acc[3] = {a0, a1, a2};
    const int b = d.bc[i];
    for (int a = 0; a < 3; ++a) {
        if (pi[a]) {
            out[a * N + i] = pv[a];
            continue;
        }
        double load = acc[a];
        if (b >= 0) {
            const BcDev& B = d.bcs[b];
            if (B.type == PD_BC_TRACTION && B.dir[a] == 1) load += B.val[a] * time_factor(B, t) / d.dx;
        }
        out[a * N + i] = load;
    }
}

// ------------------------------------------------------------------ scan

constexpr int kScanBlock = 1024;

__global__ void k_scan_block(const int64_t* __restrict__ in, int64_t* __restrict__ out, int64_t n,
                             int64_t* __restrict__ bsum) {
    __shared__ int64_t wsum[32];
    const int64_t i = blockIdx.x * (int64_t)kScanBlock + threadIdx.x;
    int64_t v = (i < n) ? in[i] : 0;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int64_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
        int64_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[w] = x;
    __syncthreads();
    if (w == 0) {
        int64_t s = wsum[lane];
        for (int o = 1; o < 32; o <<= 1) {
            int64_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        wsum[lane] = s;
    }
    __syncthreads();
    const int64_t incl = x + (w > 0 ? wsum[w - 1] : 0);
    if (i < n) out[i] = incl - v;  // exclusive
    if (threadIdx.x == kScanBlock - 1) bsum[blockIdx.x] = incl;
}

__global__ void k_scan_add(int64_t* out, int64_t n, const int64_t* __restrict__ boff) {
    const int64_t i = blockIdx.x * (int64_t)kScanBlock + threadIdx.x;
    if (i < n) out[i] += boff[blockIdx.x];
}

__global__ void k_scan_total(const int64_t* in, int64_t* out, int64_t n) {
    if (threadIdx.x == 0 && blockIdx.x == 0) out[n] = (n > 0) ? out[n - 1] + in[n - 1] : 0;
}

}  // namespace

int exclusive_scan_i64(const int64_t* in, int64_t* out, int64_t n, cudaStream_t s) {
    if (n <= 0) {
        int64_t z = 0;
        if (cudaMemcpyAsync(out, &z, sizeof(z), cudaMemcpyHostToDevice, s) != cudaSuccess) return PD_ERR_CUDA;
        return cudaStreamSynchronize(s) == cudaSuccess ? PD_OK : PD_ERR_CUDA;
    }
    const int64_t nb = (n + kScanBlock - 1) / kScanBlock;
    int64_t *bsum = nullptr, *boff = nullptr;
    if (cudaMalloc(&bsum, sizeof(int64_t) * (nb + 1)) != cudaSuccess) return PD_ERR_OOM;
    if (cudaMalloc(&boff, sizeof(int64_t) * (nb + 1)) != cudaSuccess) {
        cudaFree(bsum);
        return PD_ERR_OOM;
    }
    k_scan_block<<<(unsigned)nb, kScanBlock, 0, s>>>(in, out, n, bsum);
    int rc = PD_OK;
    if (nb > 1) {
        rc = exclusive_scan_i64(bsum, boff, nb, s);
        if (rc == PD_OK) k_scan_add<<<(unsigned)nb, kScanBlock, 0, s>>>(out, n, boff);
    }
    if (rc == PD_OK) k_scan_total<<<1, 32, 0, s>>>(in, out, n);
    if (rc == PD_OK && cudaGetLastError() != cudaSuccess) rc = PD_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) rc = PD_ERR_CUDA;
    cudaFree(bsum);
    cudaFree(boff);
    return rc;
}

void launch_static_apply_f64(const Dev& d, double t, const double* x, double* y, cudaStream_t s) {
    if (d.n == 0) return;
    if (d.sfac) k_static_apply_f64<true><<<blocks_for(d.n, 128), 128, 0, s>>>(d, t, x, y);
    else k_static_apply_f64<false><<<blocks_for(d.n, 128), 128, 0, s>>>(d, t, x, y);
}

void launch_static_apply_f32x(const Dev& d, double t, const double* x, double* y, cudaStream_t s) {
    if (d.n == 0) return;
    if (d.sfac) k_static_apply_f32x<true><<<blocks_for(d.n, 128), 128, 0, s>>>(d, t, x, y);
    else k_static_apply_f32x<false><<<blocks_for(d.n, 128), 128, 0, s>>>(d, t, x, y);
}

size_t static_nd_smem(const StencilDev& S, int R) { return nd_smem(S, R); }

void launch_static_ndiag(const StencilDev& S, int64_t n, double* D, cudaStream_t s) {
    if (n) k_static_ndiag<<<blocks_for(n, 128), 128, 0, s>>>(S, n, D);
}

void launch_static_pmask(const Dev& d, uint8_t* pm, cudaStream_t s) {
    if (d.n == 0) return;
    k_static_pmask<<<blocks_for(d.n, 256), 256, 0, s>>>(d, pm);
}

void launch_static_stencil(const Dev& d, const StencilDev& S, bool f32, const double* x, double* y, cudaStream_t s) {
    if (d.n == 0) return;
    const size_t sh = (size_t)S.ns * (sizeof(double4) + sizeof(float4) + sizeof(int4));
    const unsigned nb = blocks_for(d.n, 256);
    const bool zcol = S.ncol > 0 && S.rz >= 1 && S.rz <= 4;
    if (f32) {
        float* xm = reinterpret_cast<float*>(S.xm);
        k_static_mask<float><<<nb, 256, 0, s>>>(S.pmask, d.n, x, xm);
        if (zcol) {
            if (d.sfac) launch_zcol<float, true, 8>(d, S, x, xm, y, s);
            else launch_zcol<float, false, 8>(d, S, x, xm, y, s);
        } else if (d.sfac) {
            k_static_stencil<float, true><<<nb, 256, sh, s>>>(d, S, x, xm, y);
        } else {
            k_static_stencil<float, false><<<nb, 256, sh, s>>>(d, S, x, xm, y);
        }
    } else {
        double* xm = S.xm;
        k_static_mask<double><<<nb, 256, 0, s>>>(S.pmask, d.n, x, xm);
        if (S.ndcol > 0 && S.ndhost && !d.sfac && (S.ndr == 2 || S.ndr == 4 || S.ndr == 8) && nd_halo(S) > 0 &&
            nd_smem(S, S.ndr) <= 227 * 1024) {
            if (S.ndr == 2) launch_nd<2>(d, S, x, xm, y, s);
            else if (S.ndr == 4) launch_nd<4>(d, S, x, xm, y, s);
            else launch_nd<8>(d, S, x, xm, y, s);
        } else if (zcol) {
            if (d.sfac) launch_zcol<double, true, 4>(d, S, x, xm, y, s);
            else launch_zcol<double, false, 4>(d, S, x, xm, y, s);
        } else if (d.sfac) {
            k_static_stencil<double, true><<<nb, 256, sh, s>>>(d, S, x, xm, y);
        } else {
            k_static_stencil<double, false><<<nb, 256, sh, s>>>(d, S, x, xm, y);
        }
    }
}

void launch_static_bjacobi(const Dev& d, double* minv, cudaStream_t s) {
    if (d.n == 0) return;
    if (d.sfac) k_static_bjacobi<true><<<blocks_for(d.n, 128), 128, 0, s>>>(d, minv);
    else k_static_bjacobi<false><<<blocks_for(d.n, 128), 128, 0, s>>>(d, minv);
}

void launch_bj_apply(const double* minv, const double* r, double* z, int64_t n, cudaStream_t s) {
    if (n) k_bj_apply<<<148 * 8, 256, 0, s>>>(minv, r, z, n);
}

void launch_static_rhs(const Dev& d, double t, double* b, cudaStream_t s) {
    if (d.n == 0) return;
    if (d.sfac) k_static_rhs<true><<<blocks_for(d.n, 128), 128, 0, s>>>(d, t, b);
    else k_static_rhs<false><<<blocks_for(d.n, 128), 128, 0, s>>>(d, t, b);
}

// -------------------------------------------------------------- CG pieces

namespace {

template <typename T>
__global__ void k_dot_partial(const T* __restrict__ a, const T* __restrict__ b, int64_t n, double* __restrict__ part) {
    __shared__ double sh[256];
    double acc = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        acc += (double)a[i] * (double)b[i];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__global__ void k_dot_final(const double* __restrict__ part, int nb, double* __restrict__ out) {
    __shared__ double sh[32];
    double acc = 0.0;
    for (int k = threadIdx.x; k < nb; k += 32) acc += part[k];
    sh[threadIdx.x] = acc;
    __syncwarp();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int k = 0; k < 32; ++k) s += sh[k];
        *out = s;
    }
}

template <typename T>
__global__ void k_cg_x(T* x, T* r, const T* p, const T* q, int64_t n, const double* scal) {
    const double alpha = scal[CG_RR] / scal[CG_PQ];
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        x[i] = (T)((double)x[i] + alpha * (double)p[i]);
        r[i] = (T)((double)r[i] - alpha * (double)q[i]);
    }
}

template <typename T>
__global__ void k_cg_p(const T* r, T* p, int64_t n, const double* scal) {
    const double beta = scal[CG_RRN] / scal[CG_RR];
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = (T)((double)r[i] + beta * (double)p[i]);
}

__global__ void k_cg_swap(double* scal) {
    if (threadIdx.x == 0 && blockIdx.x == 0) scal[CG_RR] = scal[CG_RRN];
}

__global__ void k_sub(const double* a, const double* b, double* o, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        o[i] = a[i] - b[i];
}

constexpr int kStreamBlocks = 148 * 8;

}  // namespace

void launch_dot_f64(const double* a, const double* b, int64_t n, double* part, double* out, cudaStream_t s) {
    k_dot_partial<double><<<kDotBlocks, 256, 0, s>>>(a, b, n, part);
    k_dot_final<<<1, 32, 0, s>>>(part, kDotBlocks, out);
}
void launch_cg_update_x_f64(double* x, double* r, const double* p, const double* q, int64_t n, const double* scal,
                            cudaStream_t s) {
    k_cg_x<double><<<kStreamBlocks, 256, 0, s>>>(x, r, p, q, n, scal);
}
void launch_cg_update_p_f64(const double* r, double* p, int64_t n, const double* scal, cudaStream_t s) {
    k_cg_p<double><<<kStreamBlocks, 256, 0, s>>>(r, p, n, scal);
}
void launch_cg_swap(double* scal, cudaStream_t s) { k_cg_swap<<<1, 32, 0, s>>>(scal); }
void launch_sub_f64(const double* a, const double* b, double* o, int64_t n, cudaStream_t s) {
    k_sub<<<kStreamBlocks, 256, 0, s>>>(a, b, o, n);
}

}  // namespace pd
