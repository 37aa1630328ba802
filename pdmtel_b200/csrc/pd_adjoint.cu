// Adjoint (vector-Jacobian) kernels of the FP64 FGI path.
//
// Bond force of one Gauss-point evaluation (pdDataManager2.cpp:1293-1351),
// with y = xi + eta, r = |xi|, p = |y| and kappa = bE * beta * c * W:
//     f = kappa (1/r - 1/p) y,
//     df/dy = kappa [ (1/r - 1/p) I + y y^T / p^3 ]       (symmetric)
// so for an adjoint lambda of the node force,
//     dJ/dy = kappa [ (1/r - 1/p) lambda + y (y . lambda) / p^3 ],
// eta = ug_jg - u_i passes it to u_i (minus) and to the Gauss point (plus),
// and dJ/dc_ij = sum_g bE beta W (1/r - 1/p) (y . lambda).  With the pair
// spring c_ij = c_min (f_i + f_j) / 2, dJ/df_i and dJ/df_j each receive
// c_min / 2 of it.  A Gauss point whose stretch is past the critical one
// carries no force, and none of its derivative (the test itself is a step).
//
// Both halves are gathers: k_vjp_own runs over node i's family and writes
// dJ/du_i; k_vjp_partner runs over node j's family (the family relation is
// symmetric) and writes dJ/dug of j's Gauss points.  No atomics, so the
// gradient is deterministic.
#include "pd_internal.cuh"

namespace pd {

namespace {

inline unsigned blocks_for(int64_t n, int bs) { return (unsigned)((n + bs - 1) / bs); }

__device__ __forceinline__ double beta_f(double dist, double delta, double dx) {
    const double inner = delta - 0.5 * dx, outer = delta + 0.5 * dx;
    if (dist <= inner) return 1.0;
    if (dist <= outer) return (delta + 0.5 * dx - dist) / dx;
    return 0.0;
}

// p - r = eta.(2 xi + eta) / (p + r), free of cancellation at small strain
__device__ __forceinline__ double extension(double x0, double x1, double x2, double e0, double e1, double e2,
                                            double r, double p) {
    const double q = e0 * (2.0 * x0 + e0) + e1 * (2.0 * x1 + e1) + e2 * (2.0 * x2 + e2);
    return q / (p + r);
}

__device__ __forceinline__ double pair_c(const Dev& d, int64_t i, int64_t j, double* cmin) {
    const double ci = d.mats[d.mat[i]].spring, cj = d.mats[d.mat[j]].spring;
    *cmin = (cj < ci) ? cj : ci;
    return d.sfac ? *cmin * (0.5 * (d.sfac[i] + d.sfac[j])) : *cmin;
}

// u used for node i in the force of a stage: U for nodes with a boundary
// condition, the trial displacement otherwise (pdDataManager.cpp:1872-1885)
__device__ __forceinline__ void ueff(const Dev& d, const double* teU, const double* teus, int64_t i, double* u) {
    const double* s = d.bc[i] >= 0 ? teU : teus;
    u[0] = s[i];
    u[1] = s[d.n + i];
    u[2] = s[2 * d.n + i];
}

// L lanes per node (L divides 32): lane l takes the Gauss points l, l+L, ...;
// the per-node sums close with a butterfly over the L lanes (fixed order,
// so the result is deterministic).  Nodes are taken in the tiled order.
template <int L>
__device__ __forceinline__ double lane_sum(double v) {
#pragma unroll
    for (int o = L / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// one Gauss point of the bond (i, j): y = (x_j + h_g + ug_jg) - (x_i + u_i);
// returns false for a point past the critical stretch (no force)
struct PointTerms {
    double y0, y1, y2, a, q, bw;
};

__device__ __forceinline__ bool point_terms(const Dev& d, const GaussConst& G, double x0, double x1, double x2,
                                            double e0, double e1, double e2, double l0, double l1, double l2,
                                            double ecrit, double bE, PointTerms& T) {
    T.y0 = x0 + e0;
    T.y1 = x1 + e1;
    T.y2 = x2 + e2;
    // 1/r and 1/p from rsqrt (the derivative needs no bit parity with the
    // reference's IEEE square roots and divisions; the adjoint's own checks
    // hold it to 1e-10 of the oracle's gradient)
    const double r2 = x0 * x0 + x1 * x1 + x2 * x2, p2 = T.y0 * T.y0 + T.y1 * T.y1 + T.y2 * T.y2;
    const double rinv = rsqrt(r2), ip = rsqrt(p2);
    const double r = r2 * rinv, pl = p2 * ip;
    const double ext = extension(x0, x1, x2, e0, e1, e2, r, pl);
    if (ext > 0.0 && ext * rinv > ecrit) return false;
    T.bw = bE * beta_f(r, d.delta, G.dxe) * G.W;
    T.a = ext * rinv * ip;  // 1/r - 1/p
    const double yl = T.y0 * l0 + T.y1 * l1 + T.y2 * l2;
    T.q = yl * ip * ip * ip;
    return true;
}

// The same terms in FP32 (PD_OPT_ADJOINT_VJP32, on the tape of an FP32C
// forward run): the bond vector and the relative displacement are formed in
// FP64 from the tape and rounded once; 1/r, 1/p from rsqrtf; the extension
// from the cancellation-free form.  The derivative is that of the exact
// force, which the FP32 form's series approximates to FP32 rounding.  For a
// smooth adjoint the family sums of the y (y . lambda) / p^3 terms cancel to
// a first difference, so their FP32 rounding leaves about 1e-3 relative in
// the gradient (6e-3 measured on the 64x64x8 specimen with J = |U|^2 / 2).
struct PointTermsF {
    float y0, y1, y2, a, q, bw;
};

__device__ __forceinline__ float beta_ff(float dist, float delta, float dx) {
    const float inner = delta - 0.5f * dx, outer = delta + 0.5f * dx;
    if (dist <= inner) return 1.f;
    if (dist <= outer) return (outer - dist) / dx;
    return 0.f;
}

__device__ __forceinline__ bool point_terms_f(const Dev& d, const GaussConst& G, float x0, float x1, float x2,
                                              float e0, float e1, float e2, float l0, float l1, float l2,
                                              float ecrit, float bE, PointTermsF& T) {
    T.y0 = x0 + e0;
    T.y1 = x1 + e1;
    T.y2 = x2 + e2;
    const float r2 = fmaf(x0, x0, fmaf(x1, x1, x2 * x2));
    const float p2 = fmaf(T.y0, T.y0, fmaf(T.y1, T.y1, T.y2 * T.y2));
    const float rinv = rsqrtf(r2), ip = rsqrtf(p2);
    const float r = r2 * rinv, pl = p2 * ip;
    const float qx = fmaf(e0, 2.f * x0 + e0, fmaf(e1, 2.f * x1 + e1, e2 * (2.f * x2 + e2)));
    const float ext = __fdividef(qx, pl + r);
    if (ext > 0.f && ext * rinv > ecrit) return false;
    T.bw = bE * beta_ff(r, (float)d.delta, (float)G.dxe) * (float)G.W;
    T.a = ext * rinv * ip;  // 1/r - 1/p
    const float yl = fmaf(T.y0, l0, fmaf(T.y1, l1, T.y2 * l2));
    T.q = yl * ip * ip * ip;
    return true;
}

template <int L>
__global__ void __launch_bounds__(256) k_vjp_own(Dev d, const double* __restrict__ teU,
                                                 const double* __restrict__ teus, const double* __restrict__ teug,
                                                 const double* __restrict__ lamF, double* __restrict__ lam_u,
                                                 double* __restrict__ gradf) {
    extern __shared__ GaussConst sg[];
    for (int g = threadIdx.x; g < d.npt; g += blockDim.x) sg[g] = d.gc[g];
    __syncthreads();
    const int64_t N = d.n;
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t slot = t / L;
    const int lane = (int)(t % L);
    const bool live = slot < N;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, gf = 0.0;
    const int64_t i = live ? d.order[slot] : 0;
    if (live) {
        const double l0 = lamF[i], l1 = lamF[N + i], l2 = lamF[2 * N + i];
        double ui[3];
        ueff(d, teU, teus, i, ui);
        const double xi0 = d.x[i], xi1 = d.x[N + i], xi2 = d.x[2 * N + i];
        const MatDev& Mi = d.mats[d.mat[i]];
        for (int64_t p = d.arow[i]; p < d.arow[i + 1]; ++p) {
            const int64_t j = d.acol[p];
            double cmin;
            const double c = pair_c(d, i, j, &cmin);
            const double ecrit = fmin(Mi.ecrit, d.mats[d.mat[j]].ecrit);
            const double bE = 0.5 * (d.bdry[i] + d.bdry[j]);
            const double xj0 = d.x[j], xj1 = d.x[N + j], xj2 = d.x[2 * N + j];
            double gc = 0.0;
            for (int g = lane; g < d.npt; g += L) {
                const GaussConst& G = sg[g];
                const double x0 = (G.hg[0] + xj0) - xi0, x1 = (G.hg[1] + xj1) - xi1, x2 = (G.hg[2] + xj2) - xi2;
                const double* ug = teug + (int64_t)(3 * g) * N + j;
                PointTerms T;
                if (!point_terms(d, G, x0, x1, x2, ug[0] - ui[0], ug[N] - ui[1], ug[2 * N] - ui[2], l0, l1, l2,
                                 ecrit, bE, T))
                    continue;
                const double k = T.bw * c;
                a0 -= k * (T.a * l0 + T.y0 * T.q);
                a1 -= k * (T.a * l1 + T.y1 * T.q);
                a2 -= k * (T.a * l2 + T.y2 * T.q);
                gc += T.bw * T.a * (T.y0 * l0 + T.y1 * l1 + T.y2 * l2);
            }
            gf += gc * (0.5 * cmin);
        }
    }
    a0 = lane_sum<L>(a0);
    a1 = lane_sum<L>(a1);
    a2 = lane_sum<L>(a2);
    gf = lane_sum<L>(gf);
    if (live && lane == 0) {
        lam_u[i] = a0;
        lam_u[N + i] = a1;
        lam_u[2 * N + i] = a2;
        if (d.sfac) gradf[i] += gf;
    }
}

template <int L>
__global__ void __launch_bounds__(256) k_vjp_partner(Dev d, const double* __restrict__ teU,
                                                     const double* __restrict__ teus, const double* __restrict__ teug,
                                                     const double* __restrict__ lamF, double* __restrict__ lam_ug,
                                                     double* __restrict__ gradf) {
    extern __shared__ GaussConst sg[];
    for (int g = threadIdx.x; g < d.npt; g += blockDim.x) sg[g] = d.gc[g];
    __syncthreads();
    const int64_t N = d.n;
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t slot = t / L;
    const int lane = (int)(t % L);
    const bool live = slot < N;
    double gf = 0.0;
    const int64_t j = live ? d.order[slot] : 0;
    if (live) {
        const double xj0 = d.x[j], xj1 = d.x[N + j], xj2 = d.x[2 * N + j];
        const MatDev& Mj = d.mats[d.mat[j]];
        for (int g = lane; g < d.npt; g += L) {
            const GaussConst& G = sg[g];
            const double* ug = teug + (int64_t)(3 * g) * N + j;
            const double ug0 = ug[0], ug1 = ug[N], ug2 = ug[2 * N];
            const double q0 = G.hg[0] + xj0, q1 = G.hg[1] + xj1, q2 = G.hg[2] + xj2;
            double o0 = 0.0, o1 = 0.0, o2 = 0.0;
            for (int64_t p = d.arow[j]; p < d.arow[j + 1]; ++p) {
                const int64_t i = d.acol[p];
                const double l0 = lamF[i], l1 = lamF[N + i], l2 = lamF[2 * N + i];
                double ui[3];
                ueff(d, teU, teus, i, ui);
                double cmin;
                const double c = pair_c(d, i, j, &cmin);
                const double ecrit = fmin(d.mats[d.mat[i]].ecrit, Mj.ecrit);
                const double bE = 0.5 * (d.bdry[i] + d.bdry[j]);
                const double x0 = q0 - d.x[i], x1 = q1 - d.x[N + i], x2 = q2 - d.x[2 * N + i];
                PointTerms T;
                if (!point_terms(d, G, x0, x1, x2, ug0 - ui[0], ug1 - ui[1], ug2 - ui[2], l0, l1, l2, ecrit, bE,
                                 T))
                    continue;
                const double k = T.bw * c;
                o0 += k * (T.a * l0 + T.y0 * T.q);
                o1 += k * (T.a * l1 + T.y1 * T.q);
                o2 += k * (T.a * l2 + T.y2 * T.q);
                gf += T.bw * T.a * (T.y0 * l0 + T.y1 * l1 + T.y2 * l2) * (0.5 * cmin);
            }
            double* o = lam_ug + (int64_t)(3 * g) * N + j;
            o[0] = o0;
            o[N] = o1;
            o[2 * N] = o2;
        }
    }
    gf = lane_sum<L>(gf);
    if (live && lane == 0 && d.sfac) gradf[j] += gf;
}

// FP32 versions of the two VJP halves (same traversal, FP32 point terms and
// FP32 sums per lane, closed in FP64 across the lanes)
template <int L>
__global__ void __launch_bounds__(256) k_vjp_own_f32(Dev d, const double* __restrict__ teU,
                                                     const double* __restrict__ teus, const double* __restrict__ teug,
                                                     const double* __restrict__ lamF, double* __restrict__ lam_u,
                                                     double* __restrict__ gradf) {
    extern __shared__ GaussConst sg[];
    for (int g = threadIdx.x; g < d.npt; g += blockDim.x) sg[g] = d.gc[g];
    __syncthreads();
    const int64_t N = d.n;
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t slot = t / L;
    const int lane = (int)(t % L);
    const bool live = slot < N;
    float a0 = 0.f, a1 = 0.f, a2 = 0.f, gf = 0.f;
    const int64_t i = live ? d.order[slot] : 0;
    if (live) {
        const float l0 = (float)lamF[i], l1 = (float)lamF[N + i], l2 = (float)lamF[2 * N + i];
        double ui[3];
        ueff(d, teU, teus, i, ui);
        const double xi0 = d.x[i], xi1 = d.x[N + i], xi2 = d.x[2 * N + i];
        const MatDev& Mi = d.mats[d.mat[i]];
        for (int64_t p = d.arow[i]; p < d.arow[i + 1]; ++p) {
            const int64_t j = d.acol[p];
            double cmin;
            const float c = (float)pair_c(d, i, j, &cmin);
            const float ecrit = (float)fmin(Mi.ecrit, d.mats[d.mat[j]].ecrit);
            const float bE = (float)(0.5 * (d.bdry[i] + d.bdry[j]));
            const double dx0 = d.x[j] - xi0, dx1 = d.x[N + j] - xi1, dx2 = d.x[2 * N + j] - xi2;
            float gc = 0.f;
            for (int g = lane; g < d.npt; g += L) {
                const GaussConst& G = sg[g];
                const double* ug = teug + (int64_t)(3 * g) * N + j;
                PointTermsF T;
                if (!point_terms_f(d, G, (float)(G.hg[0] + dx0), (float)(G.hg[1] + dx1), (float)(G.hg[2] + dx2),
                                   (float)(ug[0] - ui[0]), (float)(ug[N] - ui[1]), (float)(ug[2 * N] - ui[2]), l0,
                                   l1, l2, ecrit, bE, T))
                    continue;
                const float k = T.bw * c;
                a0 -= k * fmaf(T.a, l0, T.y0 * T.q);
                a1 -= k * fmaf(T.a, l1, T.y1 * T.q);
                a2 -= k * fmaf(T.a, l2, T.y2 * T.q);
                gc += T.bw * T.a * fmaf(T.y0, l0, fmaf(T.y1, l1, T.y2 * l2));
            }
            gf += gc * (float)(0.5 * cmin);
        }
    }
    const double s0 = lane_sum<L>((double)a0), s1 = lane_sum<L>((double)a1), s2 = lane_sum<L>((double)a2);
    const double sf = lane_sum<L>((double)gf);
    if (live && lane == 0) {
        lam_u[i] = s0;
        lam_u[N + i] = s1;
        lam_u[2 * N + i] = s2;
        if (d.sfac) gradf[i] += sf;
    }
}

template <int L>
__global__ void __launch_bounds__(256) k_vjp_partner_f32(Dev d, const double* __restrict__ teU,
                                                         const double* __restrict__ teus,
                                                         const double* __restrict__ teug,
                                                         const double* __restrict__ lamF, double* __restrict__ lam_ug,
                                                         double* __restrict__ gradf) {
    extern __shared__ GaussConst sg[];
    for (int g = threadIdx.x; g < d.npt; g += blockDim.x) sg[g] = d.gc[g];
    __syncthreads();
    const int64_t N = d.n;
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t slot = t / L;
    const int lane = (int)(t % L);
    const bool live = slot < N;
    float gf = 0.f;
    const int64_t j = live ? d.order[slot] : 0;
    if (live) {
        const double xj0 = d.x[j], xj1 = d.x[N + j], xj2 = d.x[2 * N + j];
        const MatDev& Mj = d.mats[d.mat[j]];
        for (int g = lane; g < d.npt; g += L) {
            const GaussConst& G = sg[g];
            const double* ug = teug + (int64_t)(3 * g) * N + j;
            const double ug0 = ug[0], ug1 = ug[N], ug2 = ug[2 * N];
            const double q0 = G.hg[0] + xj0, q1 = G.hg[1] + xj1, q2 = G.hg[2] + xj2;
            float o0 = 0.f, o1 = 0.f, o2 = 0.f;
            for (int64_t p = d.arow[j]; p < d.arow[j + 1]; ++p) {
                const int64_t i = d.acol[p];
                const float l0 = (float)lamF[i], l1 = (float)lamF[N + i], l2 = (float)lamF[2 * N + i];
                double ui[3];
                ueff(d, teU, teus, i, ui);
                double cmin;
                const float c = (float)pair_c(d, i, j, &cmin);
                const float ecrit = (float)fmin(d.mats[d.mat[i]].ecrit, Mj.ecrit);
                const float bE = (float)(0.5 * (d.bdry[i] + d.bdry[j]));
                PointTermsF T;
                if (!point_terms_f(d, G, (float)(q0 - d.x[i]), (float)(q1 - d.x[N + i]), (float)(q2 - d.x[2 * N + i]),
                                   (float)(ug0 - ui[0]), (float)(ug1 - ui[1]), (float)(ug2 - ui[2]), l0, l1, l2,
                                   ecrit, bE, T))
                    continue;
                const float k = T.bw * c;
                o0 += k * fmaf(T.a, l0, T.y0 * T.q);
                o1 += k * fmaf(T.a, l1, T.y1 * T.q);
                o2 += k * fmaf(T.a, l2, T.y2 * T.q);
                gf += T.bw * T.a * fmaf(T.y0, l0, fmaf(T.y1, l1, T.y2 * l2)) * (float)(0.5 * cmin);
            }
            double* o = lam_ug + (int64_t)(3 * g) * N + j;
            o[0] = o0;
            o[N] = o1;
            o[2 * N] = o2;
        }
    }
    const double sf = lane_sum<L>((double)gf);
    if (live && lane == 0 && d.sfac) gradf[j] += sf;
}

// transpose of the MLS gather: lam_us[k] += sum over the Gauss points (j,g)
// of nodes without a boundary condition that k contributes to, of
// coeff * lam_ug[j,g].  tptr/tj/tpos: for each k, the (node j, position of k
// in j's contributor list) pairs.
__global__ void k_gather_T(Dev d, const int64_t* __restrict__ tptr, const int32_t* __restrict__ tj,
                           const int32_t* __restrict__ tpos, const double* __restrict__ lam_ug,
                           double* __restrict__ lam_us) {
    const int64_t N = d.n;
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= N) return;
    const int npt = d.npt;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    if (!d.mls) {  // every Gauss point of a node without a BC takes the node's displacement
        if (d.bc[k] >= 0) return;
        for (int g = 0; g < npt; ++g) {
            a0 += lam_ug[(int64_t)(3 * g) * N + k];
            a1 += lam_ug[(int64_t)(3 * g + 1) * N + k];
            a2 += lam_ug[(int64_t)(3 * g + 2) * N + k];
        }
        lam_us[k] += a0;
        lam_us[N + k] += a1;
        lam_us[2 * N + k] += a2;
        return;
    }
    for (int64_t e = tptr[k]; e < tptr[k + 1]; ++e) {
        const int64_t j = tj[e];
        const double* cf = d.coeff + (d.cbptr[j] + tpos[e]) * npt;
        for (int g = 0; g < npt; ++g) {
            const double c = cf[g];
            a0 += c * lam_ug[(int64_t)(3 * g) * N + j];
            a1 += c * lam_ug[(int64_t)(3 * g + 1) * N + j];
            a2 += c * lam_ug[(int64_t)(3 * g + 2) * N + j];
        }
    }
    lam_us[k] += a0;
    lam_us[N + k] += a1;
    lam_us[2 * N + k] += a2;
}

// the BC overwrite masks of UpdateNodeStatusWithBC (pdDataManager.cpp:2524-2594)
__device__ __forceinline__ bool vbuf_fixed(const Dev& d, int64_t i, int a) {
    const int b = d.bc[i];
    if (b < 0) return false;
    const BcDev& B = d.bcs[b];
    return B.dir[a] == 1 && (B.type == PD_BC_DISPL || B.type == PD_BC_VELOC || B.type == PD_BC_DISPLGRAD);
}

__device__ __forceinline__ bool u_fixed(const Dev& d, int64_t i, int a) {
    const int b = d.bc[i];
    if (b < 0) return false;
    const BcDev& B = d.bcs[b];
    return B.dir[a] == 1 && (B.type == PD_BC_DISPL || B.type == PD_BC_DISPLGRAD);
}

// adjoint of the combination step (pdDataManager.cpp:2059-2092)
__global__ void k_adj_combine(Dev d, double dt, const double* __restrict__ lUp, const double* __restrict__ lVp,
                              AdjBuf A) {
    const int64_t N = d.n;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= N) return;
    const double rho = d.mats[d.mat[i]].density;
    const bool bc = d.bc[i] >= 0;
    for (int a = 0; a < 3; ++a) {
        const int64_t r = a * N + i;
        const double lu = lUp[r], lv = lVp[r];
        A.lk1[r] = lu / 6.0;
        A.lk4[r] = lu / 6.0;
        A.lk2[r] = lu / 3.0;
        A.lk3[r] = lu / 3.0;
        A.lU[r] = u_fixed(d, i, a) ? 0.0 : lu;
        A.lV[r] = (bc ? 0.0 : -dt * d.damping * dt / rho * lu) - d.damping * dt / rho * lv;
        A.lvb[r] = lv;
        A.lu1[r] = 0.0;
    }
}

// start of a stage's adjoint: lvb += dts * lk (k = vbuf dts), the BC
// overwrite mask, lamF = lvb dts / rho
__global__ void k_adj_stage_pre(Dev d, double dts, const double* __restrict__ lk, AdjBuf A) {
    const int64_t N = d.n;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= N) return;
    const double rho = d.mats[d.mat[i]].density;
    for (int a = 0; a < 3; ++a) {
        const int64_t r = a * N + i;
        double v = A.lvb[r] + dts * lk[r];
        if (vbuf_fixed(d, i, a)) v = 0.0;
        A.lvb[r] = v;
        A.lF[r] = v * dts / rho;
    }
}

// after the force VJP of stage s >= 2: the node part goes to us (nodes
// without a BC) or to the step's input U (BC nodes, unless fixed by the
// stage-1 update); lus then receives the transposed gather
__global__ void k_adj_stage_node(Dev d, AdjBuf A) {
    const int64_t N = d.n;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= N) return;
    const bool bc = d.bc[i] >= 0;
    for (int a = 0; a < 3; ++a) {
        const int64_t r = a * N + i;
        const double l = A.lueff[r];
        if (bc) {
            A.lus[r] = 0.0;
            if (!u_fixed(d, i, a)) A.lU[r] += l;
        } else {
            A.lus[r] = l;
        }
    }
}

// us_s = u1 + alpha k_{s-1}: lu1 += lus, lk_prev += alpha lus
__global__ void k_adj_stage_post(Dev d, double alpha, double* __restrict__ lk_prev, AdjBuf A) {
    const int64_t N = d.n;
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= 3 * N) return;
    A.lu1[t] += A.lus[t];
    lk_prev[t] += alpha * A.lus[t];
}

// stage 1: the force uses the step's input U for every node and the input
// velocity buffer is V
__global__ void k_adj_stage1_end(Dev d, AdjBuf A) {
    const int64_t N = d.n;
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= 3 * N) return;
    A.lU[t] += A.lueff[t] + A.lu1[t];
    A.lV[t] += A.lvb[t];
}

}  // namespace

// lanes per node: 8 for the multi-point rules, 1 for one point; f32: the
// FP32 point terms (adjoint of the FP32-compensated form)
void launch_vjp_own(const Dev& d, const double* teU, const double* teus, const double* teug, const double* lamF,
                    double* lam_u, double* gradf, cudaStream_t s, bool f32) {
    const size_t sh = (size_t)d.npt * sizeof(GaussConst);
    const unsigned b8 = blocks_for(8 * d.n, 256), b1 = blocks_for(d.n, 256);
    if (f32) {
        if (d.npt >= 8) k_vjp_own_f32<8><<<b8, 256, sh, s>>>(d, teU, teus, teug, lamF, lam_u, gradf);
        else k_vjp_own_f32<1><<<b1, 256, sh, s>>>(d, teU, teus, teug, lamF, lam_u, gradf);
    } else {
        if (d.npt >= 8) k_vjp_own<8><<<b8, 256, sh, s>>>(d, teU, teus, teug, lamF, lam_u, gradf);
        else k_vjp_own<1><<<b1, 256, sh, s>>>(d, teU, teus, teug, lamF, lam_u, gradf);
    }
}
void launch_vjp_partner(const Dev& d, const double* teU, const double* teus, const double* teug, const double* lamF,
                        double* lam_ug, double* gradf, cudaStream_t s, bool f32) {
    const size_t sh = (size_t)d.npt * sizeof(GaussConst);
    const unsigned b8 = blocks_for(8 * d.n, 256), b1 = blocks_for(d.n, 256);
    if (f32) {
        if (d.npt >= 8) k_vjp_partner_f32<8><<<b8, 256, sh, s>>>(d, teU, teus, teug, lamF, lam_ug, gradf);
        else k_vjp_partner_f32<1><<<b1, 256, sh, s>>>(d, teU, teus, teug, lamF, lam_ug, gradf);
    } else {
        if (d.npt >= 8) k_vjp_partner<8><<<b8, 256, sh, s>>>(d, teU, teus, teug, lamF, lam_ug, gradf);
        else k_vjp_partner<1><<<b1, 256, sh, s>>>(d, teU, teus, teug, lamF, lam_ug, gradf);
    }
}
void launch_gather_T(const Dev& d, const int64_t* tptr, const int32_t* tj, const int32_t* tpos, const double* lam_ug,
                     double* lam_us, cudaStream_t s) {
    k_gather_T<<<blocks_for(d.n, 128), 128, 0, s>>>(d, tptr, tj, tpos, lam_ug, lam_us);
}
void launch_adj_combine(const Dev& d, double dt, const double* lUp, const double* lVp, const AdjBuf& A,
                        cudaStream_t s) {
    k_adj_combine<<<blocks_for(d.n, 256), 256, 0, s>>>(d, dt, lUp, lVp, A);
}
void launch_adj_stage_pre(const Dev& d, double dts, const double* lk, const AdjBuf& A, cudaStream_t s) {
    k_adj_stage_pre<<<blocks_for(d.n, 256), 256, 0, s>>>(d, dts, lk, A);
}
void launch_adj_stage_node(const Dev& d, const AdjBuf& A, cudaStream_t s) {
    k_adj_stage_node<<<blocks_for(d.n, 256), 256, 0, s>>>(d, A);
}
void launch_adj_stage_post(const Dev& d, double alpha, double* lk_prev, const AdjBuf& A, cudaStream_t s) {
    k_adj_stage_post<<<blocks_for(3 * d.n, 256), 256, 0, s>>>(d, alpha, lk_prev, A);
}
void launch_adj_stage1_end(const Dev& d, const AdjBuf& A, cudaStream_t s) {
    k_adj_stage1_end<<<blocks_for(3 * d.n, 256), 256, 0, s>>>(d, A);
}

}  // namespace pd
