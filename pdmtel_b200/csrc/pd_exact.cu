// FP64 kernels of the drop-in path.
//
// This translation unit is compiled with -fmad=false: every multiply and add
// is rounded on its own, in the order the reference's C++ evaluates it, and
// double division and square root are IEEE round-to-nearest.  One thread owns
// one node and sums its family in ascending id order, which is the order of
// the reference's loops, so the force, gather and state vectors are bit-for-
// bit those of the reference CPU path (pdDataManager.cpp:1767-2134).
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <mutex>
#include <vector>

#include "pd_internal.cuh"
#include "pd_stage.cuh"

namespace pd {

namespace {

constexpr double kMega = DBL_MAX;  // pdIntgManager.h:26
constexpr double kTiny = DBL_MIN;  // pdIntgManager.h:27

__device__ __forceinline__ double dmin(double a, double b) { return (b < a) ? b : a; }  // std::min

// pdBdryCondition*::GetTimeFactor (pdBdryConditionDispl.cpp:15, ...Veloc.cpp:15,
// ...DisplGrad.cpp:16, ...Tract.cpp:15)
__device__ __forceinline__ double time_factor(const BcDev& b, double t) {
    if (b.type == PD_BC_VELOC) return (t <= b.end_time) ? 1.0 : 0.0;
    if (b.load_type == 1.0) return (t <= b.end_time) ? t / b.end_time : 1.0;
    return 1.0;
}

// pdDataManager::CalcBetaFactor, pdDataManager3.cpp:1801-1829
__device__ __forceinline__ double beta_factor(double dist, double delta, double dx, bool cci_original) {
    double inner = delta - 0.5 * dx;
    double outer = delta + 0.5 * dx;
    if (cci_original) outer = delta;
    if (dist <= inner) return 1.0;
    if (dist > inner && dist <= outer) return (delta + 0.5 * dx - dist) / dx;
    return 0.0;
}

// ------------------------------------------------------------------ force


// p - r = (p^2 - r^2) / (p + r) with p^2 - r^2 = eta.(2 xi + eta): no
// cancellation when the strain is small (PD_PREC_FP64A)
__device__ __forceinline__ double extension(double x0, double x1, double x2, double e0, double e1, double e2,
                                            double r, double p) {
    const double q = e0 * (2.0 * x0 + e0) + e1 * (2.0 * x1 + e1) + e2 * (2.0 * x2 + e2);
    return q / (p + r);
}

// One thread per node.  FGI: the Gauss-point summation branch of
// CalcBondBasedMotionRK4 (pdDataManager.cpp:1917-1962) with the per-point
// CalcBondForceCCI (pdDataManager2.cpp:1293-1351).  CCI: the one-point
// branch (pdDataManager.cpp:1818-1866).
// Eight blocks per SM (64 registers, ~200 bytes of spill to L1): the
// evaluation is a chain of IEEE square roots and divisions, so more resident
// warps hide more of it (plate step 77 -> 64.5 ms; 6 blocks 70, 12 blocks 67).
template <bool CCI, bool ENERGY, bool SFAC, bool ACC>
__global__ void __launch_bounds__(128, 8) k_force_f64(Dev d, double dts) {
    extern __shared__ GaussConst sg[];
    for (int g = threadIdx.x; g < d.npt; g += blockDim.x) sg[g] = d.gc[g];
    __syncthreads();
    const int64_t N = d.n;
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (tid >= N) return;
    const int64_t i = d.order[tid];
    const MatDev Mi = d.mats[d.mat[i]];
    const double rho = Mi.density;
    const double b0 = Mi.grav[0] * rho, b1 = Mi.grav[1] * rho, b2 = Mi.grav[2] * rho;
    const bool bci = d.bc[i] >= 0;
    const double* src = bci ? d.U : d.us;
    const double ui0 = src[i], ui1 = src[N + i], ui2 = src[2 * N + i];
    const double xi0 = d.x[i], xi1 = d.x[N + i], xi2 = d.x[2 * N + i];
    const double bEi = d.bdry[i];
    const double sfi = SFAC ? d.sfac[i] : 0.0;
    double v0 = d.vbuf[i], v1 = d.vbuf[N + i], v2 = d.vbuf[2 * N + i];
    double eacc = ENERGY ? d.eed[i] : 0.0;
    const bool cci_orig = d.cci && !d.cci_mdf;
    const int64_t pe = d.arow[i + 1];
    for (int64_t p = d.arow[i]; p < pe; ++p) {
        const int64_t j = d.acol[p];
        const MatDev& Mj = d.mats[d.mat[j]];
        const double ecrit = dmin(Mi.ecrit, Mj.ecrit);
        double c = dmin(Mi.spring, Mj.spring);
        if (SFAC) c = c * (0.5 * (sfi + d.sfac[j]));
        const double bE = 0.5 * (bEi + d.bdry[j]);
        const double xj0 = d.x[j], xj1 = d.x[N + j], xj2 = d.x[2 * N + j];
        double F0 = 0.0, F1 = 0.0, F2 = 0.0;
        if (CCI) {
            const double* sj = (d.bc[j] >= 0) ? d.U : d.us;
            const double xv0 = xj0 - xi0, xv1 = xj1 - xi1, xv2 = xj2 - xi2;
            const double ev0 = sj[j] - ui0, ev1 = sj[N + j] - ui1, ev2 = sj[2 * N + j] - ui2;
            const double r = sqrt(xv0 * xv0 + xv1 * xv1 + xv2 * xv2);
            const double y0 = xv0 + ev0, y1 = xv1 + ev1, y2 = xv2 + ev2;
            const double pl = sqrt(y0 * y0 + y1 * y1 + y2 * y2);
            const double dxe = 2.0 * d.dx / 2.0;
            const double beta = beta_factor(r, d.delta, dxe, cci_orig);
            const double u = ACC ? extension(xv0, xv1, xv2, ev0, ev1, ev2, r, pl) : pl - r;
            const double s = u / r;
            if (u <= 0.0 || (u > 0.0 && s <= ecrit)) {
                const double t = bE * d.vol_cci * beta * c * s;
                F0 = t * y0 / pl;
                F1 = t * y1 / pl;
                F2 = t * y2 / pl;
                if (ENERGY) eacc += bE * 0.5 * (0.5 * beta * (c / r) * u * u) * 1.0;
            } else if (ENERGY) {
                eacc += 0.0;
            }
        } else {
            for (int g = 0; g < d.npt; ++g) {
                const GaussConst& G = sg[g];
                const double xv0 = (G.hg[0] + xj0) - xi0;
                const double xv1 = (G.hg[1] + xj1) - xi1;
                const double xv2 = (G.hg[2] + xj2) - xi2;
                const double* ugp = d.ug + (int64_t)(3 * g) * N + j;
                const double ev0 = ugp[0] - ui0, ev1 = ugp[N] - ui1, ev2 = ugp[2 * N] - ui2;
                const double r = sqrt(xv0 * xv0 + xv1 * xv1 + xv2 * xv2);
                const double y0 = xv0 + ev0, y1 = xv1 + ev1, y2 = xv2 + ev2;
                const double pl = sqrt(y0 * y0 + y1 * y1 + y2 * y2);
                const double beta = beta_factor(r, d.delta, G.dxe, false);
                const double u = ACC ? extension(xv0, xv1, xv2, ev0, ev1, ev2, r, pl) : pl - r;
                const double s = u / r;
                double f0 = 0.0, f1 = 0.0, f2 = 0.0;
                if (u <= 0.0 || (u > 0.0 && s <= ecrit)) {
                    const double t = bE * beta * c * s;
                    f0 = t * y0 / pl;
                    f1 = t * y1 / pl;
                    f2 = t * y2 / pl;
                    if (ENERGY) eacc += bE * 0.5 * (0.5 * beta * (c / r) * u * u) * G.pw3;
                } else if (ENERGY) {
                    eacc += 0.0;
                }
                F0 += G.W * f0;
                F1 += G.W * f1;
                F2 += G.W * f2;
            }
        }
        v0 += (F0 + b0) * dts / rho;
        v1 += (F1 + b1) * dts / rho;
        v2 += (F2 + b2) * dts / rho;
    }
    d.vbuf[i] = v0;
    d.vbuf[N + i] = v1;
    d.vbuf[2 * N + i] = v2;
    if (ENERGY) d.eed[i] = eacc;
}

// FGI with eight lanes per node: lane l evaluates the Gauss points l, l+8,
// ... of every bond; the bond's force is then summed point by point in the
// reference's order (F += W_g f_g for g = 0, 1, ...) by passing each lane's
// product along the group with shuffles, so every lane holds the same F and
// the velocity update (F + b) dt/rho per bond is the reference's, bit for bit.
// More threads than k_force_f64 for the same work: the choice for lattices
// too small to fill the GPU with one thread per node.
template <bool ENERGY, bool SFAC, bool ACC>
__global__ void __launch_bounds__(128) k_force_f64_lanes(Dev d, double dts) {
    extern __shared__ GaussConst sg[];
    for (int g = threadIdx.x; g < d.npt; g += blockDim.x) sg[g] = d.gc[g];
    __syncthreads();
    const int64_t N = d.n;
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t slot = t >> 3;
    const int lane = threadIdx.x & 7;
    if (slot >= N) return;  // whole groups of 8 leave together
    const unsigned gmask = 0xffu << (threadIdx.x & 24);
    const int64_t i = d.order[slot];
    const MatDev Mi = d.mats[d.mat[i]];
    const double rho = Mi.density;
    const double b0 = Mi.grav[0] * rho, b1 = Mi.grav[1] * rho, b2 = Mi.grav[2] * rho;
    const bool bci = d.bc[i] >= 0;
    const double* src = bci ? d.U : d.us;
    const double ui0 = src[i], ui1 = src[N + i], ui2 = src[2 * N + i];
    const double xi0 = d.x[i], xi1 = d.x[N + i], xi2 = d.x[2 * N + i];
    const double bEi = d.bdry[i];
    const double sfi = SFAC ? d.sfac[i] : 0.0;
    double v0 = d.vbuf[i], v1 = d.vbuf[N + i], v2 = d.vbuf[2 * N + i];
    double eacc = ENERGY ? d.eed[i] : 0.0;
    const int npt = d.npt;
    const int64_t pe = d.arow[i + 1];
    for (int64_t p = d.arow[i]; p < pe; ++p) {
        const int64_t j = d.acol[p];
        const MatDev& Mj = d.mats[d.mat[j]];
        const double ecrit = dmin(Mi.ecrit, Mj.ecrit);
        double c = dmin(Mi.spring, Mj.spring);
        if (SFAC) c = c * (0.5 * (sfi + d.sfac[j]));
        const double bE = 0.5 * (bEi + d.bdry[j]);
        const double xj0 = d.x[j], xj1 = d.x[N + j], xj2 = d.x[2 * N + j];
        double F0 = 0.0, F1 = 0.0, F2 = 0.0;
        for (int base = 0; base < npt; base += 8) {
            const int g = base + lane;
            double w0 = 0.0, w1 = 0.0, w2 = 0.0, el = 0.0;
            if (g < npt) {
                const GaussConst& G = sg[g];
                const double xv0 = (G.hg[0] + xj0) - xi0;
                const double xv1 = (G.hg[1] + xj1) - xi1;
                const double xv2 = (G.hg[2] + xj2) - xi2;
                const double* ugp = d.ug + (int64_t)(3 * g) * N + j;
                const double ev0 = ugp[0] - ui0, ev1 = ugp[N] - ui1, ev2 = ugp[2 * N] - ui2;
                const double r = sqrt(xv0 * xv0 + xv1 * xv1 + xv2 * xv2);
                const double y0 = xv0 + ev0, y1 = xv1 + ev1, y2 = xv2 + ev2;
                const double pl = sqrt(y0 * y0 + y1 * y1 + y2 * y2);
                const double beta = beta_factor(r, d.delta, G.dxe, false);
                const double u = ACC ? extension(xv0, xv1, xv2, ev0, ev1, ev2, r, pl) : pl - r;
                const double s = u / r;
                double f0 = 0.0, f1 = 0.0, f2 = 0.0;
                if (u <= 0.0 || (u > 0.0 && s <= ecrit)) {
                    const double tt = bE * beta * c * s;
                    f0 = tt * y0 / pl;
                    f1 = tt * y1 / pl;
                    f2 = tt * y2 / pl;
                    if (ENERGY) el = bE * 0.5 * (0.5 * beta * (c / r) * u * u) * G.pw3;
                }
                w0 = G.W * f0;
                w1 = G.W * f1;
                w2 = G.W * f2;
            }
            const int cnt = npt - base < 8 ? npt - base : 8;
            for (int l = 0; l < cnt; ++l) {
                F0 += __shfl_sync(gmask, w0, l, 8);
                F1 += __shfl_sync(gmask, w1, l, 8);
                F2 += __shfl_sync(gmask, w2, l, 8);
                if (ENERGY) eacc += __shfl_sync(gmask, el, l, 8);
            }
        }
        v0 += (F0 + b0) * dts / rho;
        v1 += (F1 + b1) * dts / rho;
        v2 += (F2 + b2) * dts / rho;
    }
    if (lane == 0) {
        d.vbuf[i] = v0;
        d.vbuf[N + i] = v1;
        d.vbuf[2 * N + i] = v2;
        if (ENERGY) d.eed[i] = eacc;
    }
}

// ----------------------------------------------------------------- gather

// One thread per (node, Gauss point): CalcIntgPointDisplRK4 (pdDataManager.cpp:
// 2402-2495) with UpdateIntgPointStatusWithBC (:2604-2703).  Nodes with a
// boundary condition keep the displacement of their unflagged directions
// (VELOC and TRACTION nodes keep all three), exactly as the reference's
// Gaussian points do.
__global__ void k_gather_f64(Dev d, const double* __restrict__ us) {
    const int64_t N = d.n;
    const double t = *d.tdev;
    const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (tid >= N * d.npt) return;
    const int64_t i = d.order[tid / d.npt];
    const int g = (int)(tid % d.npt);
    double* ug = d.ug + (int64_t)(3 * g) * N + i;
    const int b = d.bc[i];
    if (b >= 0) {
        const BcDev& B = d.bcs[b];
        const double fac = time_factor(B, t);
        const GaussConst& G = d.gc[g];
        const double q0 = G.hg[0] + d.x[i], q1 = G.hg[1] + d.x[N + i], q2 = G.hg[2] + d.x[2 * N + i];
        for (int a = 0; a < 3; ++a) {
            if (B.dir[a] != 1) continue;
            if (B.type == PD_BC_DISPL) ug[a * N] = B.val[a] * fac;
            else if (B.type == PD_BC_DISPLGRAD)
                ug[a * N] = (B.val[3 * a] * q0 + B.val[3 * a + 1] * q1 + B.val[3 * a + 2] * q2) * fac;
        }
        return;
    }
    if (d.mls) {
        const int64_t c0 = d.cbptr[i], nc = d.cbptr[i + 1] - c0;
        const double* cf = d.coeff + c0 * d.npt + g;
        const int32_t* cb = d.cbidx + c0;
        double a0 = 0.0, a1 = 0.0, a2 = 0.0;
        int64_t k = 0;
        // loads of four contributors are issued together; the sums still run
        // in contributor order
        for (; k + 4 <= nc; k += 4) {
            int64_t m[4];
            double c[4], v[4][3];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                m[u] = cb[k + u];
                c[u] = cf[(k + u) * d.npt];
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                v[u][0] = us[m[u]];
                v[u][1] = us[N + m[u]];
                v[u][2] = us[2 * N + m[u]];
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                a0 += v[u][0] * c[u];
                a1 += v[u][1] * c[u];
                a2 += v[u][2] * c[u];
            }
        }
        for (; k < nc; ++k) {
            const int64_t m = cb[k];
            const double c = cf[k * d.npt];
            a0 += us[m] * c;
            a1 += us[N + m] * c;
            a2 += us[2 * N + m] * c;
        }
        ug[0] = a0;
        ug[N] = a1;
        ug[2 * N] = a2;
    } else {
        ug[0] = us[i];
        ug[N] = us[N + i];
        ug[2 * N] = us[2 * N + i];
    }
}

// --------------------------------------------------------------- epilogue

// Per node, after the force kernel of stage `stage` (1..4): the traction load
// (project rule), UpdateNodeStatusWithBC (pdDataManager.cpp:2497-2602),
// k = vbuf*dt_s (:1977-1990) and the RK4 bookkeeping of pdDataManager::RK4
// (:2027-2092): next trial displacement, k3 += k2, and at stage 4 the
// combination, the damping and the new velocity.
__global__ void k_epilogue(Dev d, int stage, double dts, double dt) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= d.n) return;
    const double t = *d.tdev;
    if (d.energy) stage_epilogue<true>(d, i, stage, dts, dt, t);
    else stage_epilogue<false>(d, i, stage, dts, dt, t);
}

// Deterministic two-level sum of red[0..N) and red[N..2N) into red[2N], red[2N+1].
__global__ void k_energy_partial(const double* __restrict__ red, int64_t N, double* __restrict__ part) {
    __shared__ double s0[256], s1[256];
    double a = 0.0, c = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        a += red[i];
        c += red[N + i];
    }
    s0[threadIdx.x] = a;
    s1[threadIdx.x] = c;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            s0[threadIdx.x] += s0[threadIdx.x + w];
            s1[threadIdx.x] += s1[threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = s0[0];
        part[2 * blockIdx.x + 1] = s1[0];
    }
}

__global__ void k_energy_final(const double* __restrict__ part, int nb, double* __restrict__ out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double a = 0.0, c = 0.0;
        for (int k = 0; k < nb; ++k) {
            a += part[2 * k];
            c += part[2 * k + 1];
        }
        out[0] = a;
        out[1] = c;
    }
}

__global__ void k_to_soa(const double* __restrict__ aos, double* __restrict__ soa, int64_t n, int comps) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= n * comps) return;
    const int64_t i = t / comps;
    const int c = (int)(t - i * comps);
    soa[c * n + i] = aos[t];
}

// k_to_soa that also records whether any value changed (bit pattern), so a
// caller can tell a round trip of the device state from a new state
__global__ void k_to_soa_changed(const double* __restrict__ aos, double* __restrict__ soa, int64_t n, int comps,
                                 int* __restrict__ changed) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= n * comps) return;
    const int64_t i = t / comps;
    const int c = (int)(t - i * comps);
    const double v = aos[t];
    if (__double_as_longlong(soa[c * n + i]) != __double_as_longlong(v)) *changed = 1;
    soa[c * n + i] = v;
}

__global__ void k_to_aos(const double* __restrict__ soa, double* __restrict__ aos, int64_t n, int comps) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= n * comps) return;
    const int64_t i = t / comps;
    const int c = (int)(t - i * comps);
    aos[t] = soa[c * n + i];
}

__global__ void k_fill(double* p, double v, int64_t n) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t < n) p[t] = v;
}

inline unsigned blocks_for(int64_t n, int bs) { return (unsigned)((n + bs - 1) / bs); }

}  // namespace

void launch_force_f64(const Dev& d, double dts, cudaStream_t s) {
    if (d.n == 0) return;
    if (d.ai) {
        launch_ai_force(d, dts, s);
        return;
    }
    const int bs = 128;
    size_t sh = (size_t)d.npt * sizeof(GaussConst);
    unsigned nb = blocks_for(d.n, bs);
    const bool sf = d.sfac != nullptr;
    if (!d.cci && d.npt >= 8 && d.n < d.f64_lanes_below) {
        const unsigned nb8 = blocks_for(8 * d.n, bs);
#define PD_FORCE_L(E, S)                                                                  \
    do {                                                                                  \
        if (d.acc_stretch) k_force_f64_lanes<E, S, true><<<nb8, bs, sh, s>>>(d, dts);    \
        else k_force_f64_lanes<E, S, false><<<nb8, bs, sh, s>>>(d, dts);                 \
    } while (0)
        if (d.energy) { if (sf) PD_FORCE_L(true, true); else PD_FORCE_L(true, false); }
        else { if (sf) PD_FORCE_L(false, true); else PD_FORCE_L(false, false); }
#undef PD_FORCE_L
        return;
    }
#define PD_FORCE(C, E, S)                                                     \
    do {                                                                      \
        if (d.acc_stretch) k_force_f64<C, E, S, true><<<nb, bs, sh, s>>>(d, dts); \
        else k_force_f64<C, E, S, false><<<nb, bs, sh, s>>>(d, dts);          \
    } while (0)
    if (d.cci) {
        if (d.energy) { if (sf) PD_FORCE(true, true, true); else PD_FORCE(true, true, false); }
        else { if (sf) PD_FORCE(true, false, true); else PD_FORCE(true, false, false); }
    } else {
        if (d.energy) { if (sf) PD_FORCE(false, true, true); else PD_FORCE(false, true, false); }
        else { if (sf) PD_FORCE(false, false, true); else PD_FORCE(false, false, false); }
    }
#undef PD_FORCE
}

void launch_gather_f64(const Dev& d, const double* us, cudaStream_t s) {
    if (d.ai) {
        launch_ai_gather(d, us, s);
        return;
    }
    if (d.cci || d.n == 0) return;
    const int bs = 256;
    k_gather_f64<<<blocks_for(d.n * d.npt, bs), bs, 0, s>>>(d, us);
}

void launch_epilogue(const Dev& d, int stage, double dts, double dt, cudaStream_t s) {
    if (d.n == 0) return;
    const int bs = 256;
    k_epilogue<<<blocks_for(d.n, bs), bs, 0, s>>>(d, stage, dts, dt);
}

// t += dt on the device, as pdSolve.cpp:61 advances currentTime
__global__ void k_advance_time(double* t, double dt) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *t = *t + dt;
}

void launch_advance_time(double* t, double dt, cudaStream_t s) { k_advance_time<<<1, 32, 0, s>>>(t, dt); }

void launch_energy_reduce(const Dev& d, cudaStream_t s) {
    const int nb = 148;
    double* part = d.red + 2 * d.n + 2;
    k_energy_partial<<<nb, 256, 0, s>>>(d.red, d.n, part);
    k_energy_final<<<1, 32, 0, s>>>(part, nb, d.red + 2 * d.n);
}

// ============================================================ MLS setup
//
// InitIntegrationPoint (pdDataManager2.cpp:118-256) on the device: the
// contributor lists and the coefficients of every Gauss point, in the
// reference's operation order (this unit is compiled with -fmad=false).  The
// one difference: the spline weight's d^3 and d^4, which the reference takes
// from glibc's pow, are rounded once here (Dekker's exact product, formed with
// FMA), and glibc's pow is off the correctly rounded value for about 4 in
// 10,000 arguments; through the ill-conditioned moment matrix (global
// coordinates) such a weight moves the coefficients by round-off amplified
// like the reference's own (1e-10..1e-5 of the largest coefficient).

__device__ __forceinline__ double cube_rn(double d) {
    const double p = d * d, ep = fma(d, d, -p);  // d^2 = p + ep exactly
    const double h = p * d, eh = fma(p, d, -h);  // p d = h + eh exactly
    return h + (eh + ep * d);
}

__device__ __forceinline__ double quart_rn(double d) {
    const double p = d * d, ep = fma(d, d, -p);
    const double q = p * p, eq = fma(p, p, -q);  // d^4 = q + eq + 2 p ep + ep^2
    return q + (eq + 2.0 * p * ep);
}

// quadratic basis in global coordinates, pdDataManager2.cpp:1547-1563
__device__ __forceinline__ void mls_basis(double q0, double q1, double q2, double* p) {
    p[0] = 1.0;
    p[1] = q0;
    p[2] = q1;
    p[3] = q2;
    p[4] = q0 * q1;
    p[5] = q0 * q2;
    p[6] = q1 * q2;
    p[7] = q0 * q0;
    p[8] = q1 * q1;
    p[9] = q2 * q2;
}

// quartic spline of |q - node| / rw, pdDataManager2.cpp:1565-1578
__device__ __forceinline__ double mls_weight(double n0, double n1, double n2, double q0, double q1, double q2,
                                             double rw) {
    const double e1 = q0 - n0, e2 = q1 - n1, e3 = q2 - n2;
    const double r = sqrt(e1 * e1 + e2 * e2 + e3 * e3);
    const double d = r / rw;
    if (d > 1.0) return 0.0;
    return (1 - 6.0 * d * d + 8.0 * cube_rn(d) - 3.0 * quart_rn(d));
}

// contributors: the node, then its family members (ascending id) within rw,
// or within 1.5 rw when fewer than 10 qualify (pdDataManager2.cpp:118-171)
template <bool FILL>
__global__ void k_mls_contrib(Dev d, const double* __restrict__ xm, double rw, int64_t* __restrict__ cnt,
                              const int64_t* __restrict__ cbptr, int32_t* __restrict__ cbidx) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= d.n) return;
    const int64_t N = d.n;
    const double x0 = xm[i], x1 = xm[N + i], x2 = xm[2 * N + i];
    double radius = rw;
    int64_t c = 1;
    for (int pass = 0; pass < 2; ++pass) {
        radius = pass == 0 ? rw : rw * 1.5;
        c = 1;
        for (int64_t p = d.frow[i]; p < d.frow[i + 1]; ++p) {
            const int64_t j = d.fcol[p];
            const double d1 = xm[j] - x0, d2 = xm[N + j] - x1, d3 = xm[2 * N + j] - x2;
            if (sqrt(d1 * d1 + d2 * d2 + d3 * d3) <= radius) ++c;
        }
        if (c >= 10) break;
    }
    if (!FILL) {
        cnt[i] = c;
        return;
    }
    int64_t o = cbptr[i];
    cbidx[o++] = (int32_t)i;
    for (int64_t p = d.frow[i]; p < d.frow[i + 1]; ++p) {
        const int64_t j = d.fcol[p];
        const double d1 = xm[j] - x0, d2 = xm[N + j] - x1, d3 = xm[2 * N + j] - x2;
        if (sqrt(d1 * d1 + d2 * d2 + d3 * d3) <= radius) cbidx[o++] = (int32_t)j;
    }
}

// One thread per (node, Gauss point): the 10x10 moment matrix sum_k w_k p_k
// p_k^T (held in shared memory, entry-major so that a warp's accesses hit
// distinct banks), the full-pivot Gauss-Jordan solve of pdMatrix::Gauss
// (pdMatrix.cpp:251-391) for A s = p(x_g), and coeff_k = w_k p_k^T s, laid
// out [node][contributor][point].  A singular matrix records its node in *bad.
__global__ void __launch_bounds__(128) k_mls_coeff(Dev d, const double* __restrict__ xm, double rw,
                                                   const double* __restrict__ absc, int n1,
                                                   const int64_t* __restrict__ cbptr,
                                                   const int32_t* __restrict__ cbidx, double* __restrict__ coeff,
                                                   unsigned long long* __restrict__ bad) {
    extern __shared__ double smA[];
    const int bs = blockDim.x, tl = threadIdx.x;
    const int npt = n1 * n1 * n1;
    const int64_t t = blockIdx.x * (int64_t)bs + tl;
    if (t >= d.n * npt) return;
    const int64_t N = d.n;
    const int64_t i = t / npt;
    const int g = (int)(t - i * npt);
    const int gi = g / (n1 * n1), gj = (g / n1) % n1, gk = g % n1;
    const double q0 = 0.5 * d.dx * absc[gi] + xm[i];
    const double q1 = 0.5 * d.dx * absc[gj] + xm[N + i];
    const double q2 = 0.5 * d.dx * absc[gk] + xm[2 * N + i];
#define PD_A(r, c) smA[((r) * 10 + (c)) * bs + tl]
    for (int k = 0; k < 100; ++k) smA[k * bs + tl] = 0.0;
    const int64_t b = cbptr[i], nc = cbptr[i + 1] - b;
    for (int64_t k = 0; k < nc; ++k) {
        const int64_t m = cbidx[b + k];
        double e[10];
        mls_basis(xm[m], xm[N + m], xm[2 * N + m], e);
        const double w = mls_weight(xm[m], xm[N + m], xm[2 * N + m], q0, q1, q2, rw);
        for (int r = 0; r < 10; ++r) {
            const double wr = w * e[r];
            for (int c = 0; c < 10; ++c) PD_A(r, c) = PD_A(r, c) + wr * e[c];
        }
    }
    double s[10];
    mls_basis(q0, q1, q2, s);
    int piv[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    bool ok = true;
    for (int step = 0; step < 10 && ok; ++step) {
        double big = 0.0;
        int prow = 0, pcol = 0;
        for (int r = 0; r < 10 && ok; ++r) {
            if (piv[r] == 1) continue;
            for (int c = 0; c < 10; ++c) {
                if (piv[c] == 0) {
                    if (fabs(PD_A(r, c)) >= big) {
                        big = fabs(PD_A(r, c));
                        prow = r;
                        pcol = c;
                    }
                } else if (piv[c] > 1) {
                    ok = false;
                    break;
                }
            }
        }
        if (!ok) break;
        ++piv[pcol];
        if (prow != pcol) {
            for (int c = 0; c < 10; ++c) {
                const double tmp = PD_A(prow, c);
                PD_A(prow, c) = PD_A(pcol, c);
                PD_A(pcol, c) = tmp;
            }
            const double tmp = s[prow];
            s[prow] = s[pcol];
            s[pcol] = tmp;
        }
        if (PD_A(pcol, pcol) == 0.0) {
            ok = false;
            break;
        }
        const double inv = 1.0 / PD_A(pcol, pcol);
        PD_A(pcol, pcol) = 1.0;
        for (int c = 0; c < 10; ++c) PD_A(pcol, c) = PD_A(pcol, c) * inv;
        s[pcol] = s[pcol] * inv;
        for (int r = 0; r < 10; ++r) {
            if (r == pcol) continue;
            const double mm = PD_A(r, pcol);
            PD_A(r, pcol) = 0.0;
            for (int c = 0; c < 10; ++c) PD_A(r, c) = PD_A(r, c) - PD_A(pcol, c) * mm;
            s[r] = s[r] + -mm * s[pcol];
        }
    }
#undef PD_A
    if (!ok) {
        atomicMin(bad, (unsigned long long)i);
        for (int64_t k = 0; k < nc; ++k) coeff[(b + k) * npt + g] = 0.0;
        return;
    }
    for (int64_t k = 0; k < nc; ++k) {
        const int64_t m = cbidx[b + k];
        double e[10];
        mls_basis(xm[m], xm[N + m], xm[2 * N + m], e);
        const double w = mls_weight(xm[m], xm[N + m], xm[2 * N + m], q0, q1, q2, rw);
        double sum = 0.0;
        for (int r = 0; r < 10; ++r) sum += (e[r] * w) * s[r];
        coeff[(b + k) * npt + g] = sum;
    }
}

// partition-of-unity defect sum_k c_k - 1 per (node, point), and the FP32
// copy of the coefficients
__global__ void k_mls_finish(Dev d, int npt, const int64_t* __restrict__ cbptr, const double* __restrict__ coeff,
                             float* __restrict__ coeff32, float* __restrict__ csum) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= d.n * npt) return;
    const int64_t i = t / npt;
    const int g = (int)(t - i * npt);
    double sum = 0.0;
    for (int64_t k = cbptr[i]; k < cbptr[i + 1]; ++k) {
        const double v = coeff[k * npt + g];
        coeff32[k * npt + g] = (float)v;
        sum += v;
    }
    csum[t] = (float)(sum - 1.0);
}

int mls_setup(const Dev& d, const double* xm, double rw, const double* absc, int n1, int64_t* cnt, int64_t* cbptr,
              int32_t** cbidx, double** coeff, float** coeff32, float** csum, int64_t* total, int64_t* bad_node,
              void* (*alloc)(void*, size_t), void* actx, cudaStream_t s) {
    const int64_t N = d.n;
    const int npt = n1 * n1 * n1;
    *bad_node = -1;
    if (N == 0) return PD_OK;
    k_mls_contrib<false><<<(unsigned)((N + 127) / 128), 128, 0, s>>>(d, xm, rw, cnt, nullptr, nullptr);
    if (exclusive_scan_i64(cnt, cbptr, N, s) != PD_OK) return PD_ERR_CUDA;
    if (cudaMemcpyAsync(total, cbptr + N, sizeof(int64_t), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return PD_ERR_CUDA;
    const int64_t T = *total;
    *cbidx = (int32_t*)alloc(actx, sizeof(int32_t) * (size_t)std::max<int64_t>(T, 1));
    *coeff = (double*)alloc(actx, sizeof(double) * (size_t)std::max<int64_t>(T * npt, 1));
    *coeff32 = (float*)alloc(actx, sizeof(float) * (size_t)std::max<int64_t>(T * npt, 1));
    *csum = (float*)alloc(actx, sizeof(float) * (size_t)(N * npt));
    if (!*cbidx || !*coeff || !*coeff32 || !*csum) return PD_ERR_OOM;
    k_mls_contrib<true><<<(unsigned)((N + 127) / 128), 128, 0, s>>>(d, xm, rw, nullptr, cbptr, *cbidx);
    unsigned long long* dbad = reinterpret_cast<unsigned long long*>(cnt);  // the counts are no longer needed
    const unsigned long long none = ~0ull;
    if (cudaMemcpyAsync(dbad, &none, sizeof none, cudaMemcpyHostToDevice, s) != cudaSuccess) return PD_ERR_CUDA;
    const int bs = 128;
    const size_t smem = sizeof(double) * 100 * bs;
    if (cudaFuncSetAttribute(k_mls_coeff, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return PD_ERR_CUDA;
    k_mls_coeff<<<(unsigned)((N * npt + bs - 1) / bs), bs, smem, s>>>(d, xm, rw, absc, n1, cbptr, *cbidx, *coeff,
                                                                      dbad);
    k_mls_finish<<<(unsigned)((N * npt + 255) / 256), 256, 0, s>>>(d, npt, cbptr, *coeff, *coeff32, *csum);
    unsigned long long hb = none;
    if (cudaMemcpyAsync(&hb, dbad, sizeof hb, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return PD_ERR_CUDA;
    if (hb != none) {
        *bad_node = (int64_t)hb;
        return PD_ERR_SINGULAR;
    }
    return cudaGetLastError() == cudaSuccess ? PD_OK : PD_ERR_CUDA;
}

void launch_to_soa(const double* aos, double* soa, int64_t n, int comps, cudaStream_t s) {
    if (n == 0) return;
    k_to_soa<<<blocks_for(n * comps, 256), 256, 0, s>>>(aos, soa, n, comps);
}

void launch_to_soa_changed(const double* aos, double* soa, int64_t n, int comps, int* changed, cudaStream_t s) {
    if (n == 0) return;
    k_to_soa_changed<<<blocks_for(n * comps, 256), 256, 0, s>>>(aos, soa, n, comps, changed);
}

void launch_to_aos(const double* soa, double* aos, int64_t n, int comps, cudaStream_t s) {
    if (n == 0) return;
    k_to_aos<<<blocks_for(n * comps, 256), 256, 0, s>>>(soa, aos, n, comps);
}

void launch_fill(double* p, double v, int64_t n, cudaStream_t s) {
    if (n == 0) return;
    k_fill<<<blocks_for(n, 256), 256, 0, s>>>(p, v, n);
}

// ============================================================ bond search

namespace {

__device__ __forceinline__ double shortest_between(double v, double lo, double hi, double tol) {
    if (v < lo - tol) return fabs(v - lo);
    if (v > hi + tol) return fabs(v - hi);
    return 0.0;
}

__device__ __forceinline__ double longest_between(double v, double lo, double hi, double tol) {
    if (v < lo - tol) return fabs(v - hi);
    if (v > hi + tol) return fabs(v - lo);
    if (v > 0.5 * (hi + lo)) return fabs(v - lo);
    return fabs(v - hi);
}

// pdDataManager::CalcDistanceToFace, pdDataManager3.cpp:1573-1661
__device__ void dist_to_face(int nrm, double xf, const double* pi, const double* pj, double dx, double* dmn,
                             double* dmx) {
    const double tol = 1e-4 * dx;
    const int n1 = nrm == 1, n2 = nrm == 2, n3 = nrm == 3;
    const double xi1 = pi[0], xi2 = pi[1], xi3 = pi[2];
    const double xj1 = pj[0], xj2 = pj[1], xj3 = pj[2];
    if (fabs((xi1 - xj1) * n1 + (xi2 - xj2) * n2 + (xi3 - xj3) * n3) < tol) {
        *dmn = kMega;
        *dmx = kTiny;
        return;
    }
    const double x1lo = xj1 - 0.5 * dx, x1hi = xj1 + 0.5 * dx;
    const double x2lo = xj2 - 0.5 * dx, x2hi = xj2 + 0.5 * dx;
    const double x3lo = xj3 - 0.5 * dx, x3hi = xj3 + 0.5 * dx;
    const double x_i = xi1 * n1 + xi2 * n2 + xi3 * n3;
    const double x_j = xj1 * n1 + xj2 * n2 + xj3 * n3;
    const double fac = (xf - x_i) / (x_j - x_i);
    const double x1int = xi1 + fac * (xj1 - xi1);
    const double x2int = xi2 + fac * (xj2 - xi2);
    const double x3int = xi3 + fac * (xj3 - xi3);
    if (x1int > x1lo - tol && x1int < x1hi + tol && x2int > x2lo - tol && x2int < x2hi + tol && x3int > x3lo - tol &&
        x3int < x3hi + tol) {
        const double f1 = (1 - n1) * xi1 + n1 * xf;
        const double f2 = (1 - n2) * xi2 + n2 * xf;
        const double f3 = (1 - n3) * xi3 + n3 * xf;
        const double s1 = (1 - n1) * shortest_between(f1, x1lo, x1hi, tol);
        const double s2 = (1 - n2) * shortest_between(f2, x2lo, x2hi, tol);
        const double s3 = (1 - n3) * shortest_between(f3, x3lo, x3hi, tol);
        const double l1 = (1 - n1) * longest_between(f1, x1lo, x1hi, tol);
        const double l2 = (1 - n2) * longest_between(f2, x2lo, x2hi, tol);
        const double l3 = (1 - n3) * longest_between(f3, x3lo, x3hi, tol);
        const double ffs = sqrt(s1 * s1 + s2 * s2 + s3 * s3);
        const double ffl = sqrt(l1 * l1 + l2 * l2 + l3 * l3);
        const double itf = sqrt((f1 - xi1) * (f1 - xi1) + (f2 - xi2) * (f2 - xi2) + (f3 - xi3) * (f3 - xi3));
        *dmn = sqrt(ffs * ffs + itf * itf);
        *dmx = sqrt(ffl * ffl + itf * itf);
        return;
    }
    *dmn = kMega;
    *dmx = kTiny;
}

// InitBond's membership test for the pair (a < b): the rough distance
// reject of pdDataManager2.cpp:34-38, then CalcDistanceToCube's minimum
// (pdDataManager3.cpp:637-685) against horizon + tolerance.
__device__ bool pair_bonded(const double* pa, const double* pb, double dx, double delta, double tol, double* dist) {
    const double d1 = pb[0] - pa[0], d2 = pb[1] - pa[1], d3 = pb[2] - pa[2];
    *dist = sqrt(d1 * d1 + d2 * d2 + d3 * d3);
    if (delta < *dist - 1.5 * dx) return false;
    double mn = kMega, a, b;
    for (int ax = 0; ax < 3; ++ax) {
        dist_to_face(ax + 1, pb[ax] - 0.5 * dx, pa, pb, dx, &a, &b);
        mn = dmin(mn, a);
        dist_to_face(ax + 1, pb[ax] + 0.5 * dx, pa, pb, dx, &a, &b);
        mn = dmin(mn, a);
    }
    return mn < delta + tol;
}

// Project rule for pdSlit (pdSlit.h:6-10 fixes only the keyword): the segment
// from the lower-id to the higher-id node crosses the rectangle.
__device__ bool slit_crosses(const double* s, const double* a, const double* b) {
    int nrm = 0;
    double ext = s[1] - s[0];
    for (int k = 1; k < 3; ++k)
        if (s[2 * k + 1] - s[2 * k] < ext) {
            ext = s[2 * k + 1] - s[2 * k];
            nrm = k;
        }
    const double c = 0.5 * (s[2 * nrm] + s[2 * nrm + 1]);
    const double da = a[nrm] - c, db = b[nrm] - c;
    if (!((da < 0.0 && db > 0.0) || (da > 0.0 && db < 0.0))) return false;
    const double t = (c - a[nrm]) / (b[nrm] - a[nrm]);
    for (int k = 0; k < 3; ++k) {
        if (k == nrm) continue;
        const double p = a[k] + t * (b[k] - a[k]);
        if (p < s[2 * k] || p > s[2 * k + 1]) return false;
    }
    return true;
}

struct SearchArgs {
    const double* x;  // [3][N]
    int64_t n;
    double dx, delta, tol;
    SearchGrid g;
    const int32_t* cell_rank;  // linear cell -> Morton rank
    const int64_t* cstart;     // [ncell+1] by rank
    const int32_t* sorted;     // nodes ordered by Morton rank of their cell
    int nslit;
    const double* slits;
};

__device__ __forceinline__ void load_x(const SearchArgs& A, int64_t i, double* p) {
    p[0] = A.x[i];
    p[1] = A.x[A.n + i];
    p[2] = A.x[2 * A.n + i];
}

__device__ __forceinline__ int64_t cell_coord(const SearchArgs& A, double v, int a) {
    int64_t c = (int64_t)floor((v - A.g.lo[a]) / A.g.h);
    if (c < 0) c = 0;
    if (c >= A.g.nc[a]) c = A.g.nc[a] - 1;
    return c;
}

__global__ void k_cell_count(SearchArgs A, int32_t* node_rank, int64_t* cnt) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= A.n) return;
    double p[3];
    load_x(A, i, p);
    const int64_t cx = cell_coord(A, p[0], 0), cy = cell_coord(A, p[1], 1), cz = cell_coord(A, p[2], 2);
    const int32_t r = A.cell_rank[(cz * A.g.nc[1] + cy) * A.g.nc[0] + cx];
    node_rank[i] = r;
    atomicAdd((unsigned long long*)&cnt[r], 1ull);
}

__global__ void k_cell_scatter(SearchArgs A, const int32_t* node_rank, const int64_t* cstart, int64_t* fillc,
                               int32_t* sorted) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= A.n) return;
    const int32_t r = node_rank[i];
    const int64_t pos = (int64_t)atomicAdd((unsigned long long*)&fillc[r], 1ull);
    sorted[cstart[r] + pos] = (int32_t)i;
}

// One warp per node (taken in Morton order of the cells so that neighbouring
// warps scan overlapping cells).  PASS 0 counts family and unbroken entries
// and the minimum bond length; PASS 1 collects the family into shared
// memory, orders it by id and writes both CSRs.
template <int PASS>
__global__ void k_search(SearchArgs A, int64_t* cnt_full, int64_t* cnt_act, unsigned long long* min_bits,
                         unsigned long long* max_cnt, const int64_t* frow, int32_t* fcol, uint8_t* fbroken,
                         const int64_t* arow, int32_t* acol, int cap) {
    extern __shared__ int32_t sbuf[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    if (w >= A.n) return;
    int32_t* buf = sbuf + (size_t)wib * cap;
    uint8_t* brk = (uint8_t*)(sbuf + (size_t)(blockDim.x >> 5) * cap) + (size_t)wib * cap;
    const int64_t i = A.sorted[w];
    double pi[3];
    load_x(A, i, pi);
    const int64_t cx = cell_coord(A, pi[0], 0), cy = cell_coord(A, pi[1], 1), cz = cell_coord(A, pi[2], 2);
    int64_t nfull = 0, nact = 0;
    double mb = A.delta;
    for (int64_t dz = -1; dz <= 1; ++dz) {
        const int64_t qz = cz + dz;
        if (qz < 0 || qz >= A.g.nc[2]) continue;
        for (int64_t dy = -1; dy <= 1; ++dy) {
            const int64_t qy = cy + dy;
            if (qy < 0 || qy >= A.g.nc[1]) continue;
            for (int64_t dxc = -1; dxc <= 1; ++dxc) {
                const int64_t qx = cx + dxc;
                if (qx < 0 || qx >= A.g.nc[0]) continue;
                const int32_t r = A.cell_rank[(qz * A.g.nc[1] + qy) * A.g.nc[0] + qx];
                const int64_t s0 = A.cstart[r], s1 = A.cstart[r + 1];
                for (int64_t s = s0; s < s1; s += 32) {
                    bool hit = false, br = false;
                    int64_t j = -1;
                    if (s + lane < s1) {
                        j = A.sorted[s + lane];
                        if (j != i) {
                            double pj[3], dist;
                            load_x(A, j, pj);
                            const double* pa = (i < j) ? pi : pj;
                            const double* pb = (i < j) ? pj : pi;
                            hit = pair_bonded(pa, pb, A.dx, A.delta, A.tol, &dist);
                            if (hit) {
                                if (i < j) mb = dmin(mb, dist);
                                for (int k = 0; k < A.nslit; ++k) br = br || slit_crosses(A.slits + 6 * k, pa, pb);
                            }
                        }
                    }
                    const unsigned hm = __ballot_sync(0xffffffffu, hit);
                    const unsigned bm = __ballot_sync(0xffffffffu, hit && !br);
                    if (PASS == 1 && hit) {
                        const int slot = (int)nfull + __popc(hm & ((1u << lane) - 1u));
                        if (slot < cap) {
                            buf[slot] = (int32_t)j;
                            brk[slot] = br ? 1 : 0;
                        }
                    }
                    nfull += __popc(hm);
                    nact += __popc(bm);
                }
            }
        }
    }
    if (PASS == 0) {
        for (int o = 16; o > 0; o >>= 1) mb = dmin(mb, __shfl_xor_sync(0xffffffffu, mb, o));
        if (lane == 0) {
            cnt_full[i] = nfull;
            cnt_act[i] = nact;
            atomicMin(min_bits, (unsigned long long)__double_as_longlong(mb));
            atomicMax(max_cnt, (unsigned long long)nfull);
        }
        return;
    }
    __syncwarp();
    const int nf = (int)(nfull < cap ? nfull : cap);
    const int64_t fo = frow[i], ao = arow[i];
    for (int e = lane; e < nf; e += 32) {
        const int32_t v = buf[e];
        int rk = 0, ra = 0;
        for (int k = 0; k < nf; ++k) {
            const int32_t o = buf[k];
            if (o < v) {
                ++rk;
                ra += brk[k] ? 0 : 1;
            }
        }
        fcol[fo + rk] = v;
        fbroken[fo + rk] = brk[e];
        if (!brk[e]) acol[ao + ra] = v;
    }
}

}  // namespace

int bond_search(const Dev& d, const SearchGrid& g, const int32_t* cell_rank, int64_t ncell, int nslit,
                const double* slits_dev, int64_t** frow_o, int32_t** fcol_o, uint8_t** fbroken_o, int64_t** arow_o,
                int32_t** acol_o, int64_t* nh, int64_t* nb, double* min_bond, cudaStream_t s) {
    const int64_t N = d.n;
    SearchArgs A;
    A.x = d.x;
    A.n = N;
    A.dx = d.dx;
    A.delta = d.delta;
    A.tol = 1.0e-4 * d.dx;
    A.g = g;
    A.cell_rank = cell_rank;
    A.nslit = nslit;
    A.slits = slits_dev;
    int32_t *node_rank = nullptr, *sorted = nullptr;
    int64_t *ccnt = nullptr, *cstart = nullptr, *fillc = nullptr, *cf = nullptr, *ca = nullptr;
    int64_t *frow = nullptr, *arow = nullptr;
    unsigned long long* scal = nullptr;
    int32_t *fcol = nullptr, *acol = nullptr;
    uint8_t* fbr = nullptr;
    int rc = PD_OK;
    auto cleanup = [&]() {
        cudaFree(node_rank); cudaFree(sorted); cudaFree(ccnt); cudaFree(cstart); cudaFree(fillc);
        cudaFree(cf); cudaFree(ca); cudaFree(scal);
    };
#define PD_S_TRY(expr)                                                        \
    do {                                                                      \
        cudaError_t _e = (expr);                                              \
        if (_e != cudaSuccess) {                                              \
            rc = fail_cuda(_e, #expr, __FILE__, __LINE__);                    \
            cleanup(); cudaFree(frow); cudaFree(arow); cudaFree(fcol);        \
            cudaFree(acol); cudaFree(fbr);                                    \
            return rc;                                                        \
        }                                                                     \
    } while (0)
    PD_S_TRY(cudaMalloc(&node_rank, sizeof(int32_t) * (N + 1)));
    PD_S_TRY(cudaMalloc(&sorted, sizeof(int32_t) * (N + 1)));
    PD_S_TRY(cudaMalloc(&ccnt, sizeof(int64_t) * (ncell + 1)));
    PD_S_TRY(cudaMalloc(&cstart, sizeof(int64_t) * (ncell + 1)));
    PD_S_TRY(cudaMalloc(&fillc, sizeof(int64_t) * (ncell + 1)));
    PD_S_TRY(cudaMalloc(&cf, sizeof(int64_t) * (N + 1)));
    PD_S_TRY(cudaMalloc(&ca, sizeof(int64_t) * (N + 1)));
    PD_S_TRY(cudaMalloc(&frow, sizeof(int64_t) * (N + 1)));
    PD_S_TRY(cudaMalloc(&arow, sizeof(int64_t) * (N + 1)));
    PD_S_TRY(cudaMalloc(&scal, sizeof(unsigned long long) * 2));
    PD_S_TRY(cudaMemsetAsync(ccnt, 0, sizeof(int64_t) * (ncell + 1), s));
    PD_S_TRY(cudaMemsetAsync(fillc, 0, sizeof(int64_t) * (ncell + 1), s));
    unsigned long long init[2] = {(unsigned long long)__builtin_bit_cast(unsigned long long, d.delta), 0ull};
    PD_S_TRY(cudaMemcpyAsync(scal, init, sizeof(init), cudaMemcpyHostToDevice, s));
    const int bs = 256;
    if (N > 0) {
        k_cell_count<<<blocks_for(N, bs), bs, 0, s>>>(A, node_rank, ccnt);
        PD_S_TRY(cudaGetLastError());
    }
    if (exclusive_scan_i64(ccnt, cstart, ncell, s) != PD_OK) { cleanup(); return fail(PD_ERR_CUDA, "scan failed"); }
    if (N > 0) {
        k_cell_scatter<<<blocks_for(N, bs), bs, 0, s>>>(A, node_rank, cstart, fillc, sorted);
        PD_S_TRY(cudaGetLastError());
    }
    A.cstart = cstart;
    A.sorted = sorted;
    const int wpb = 4;  // warps per block
    if (N > 0) {
        k_search<0><<<blocks_for(N * 32, 32 * wpb), 32 * wpb, 0, s>>>(A, cf, ca, scal, scal + 1, nullptr, nullptr,
                                                                      nullptr, nullptr, nullptr, 0);
        PD_S_TRY(cudaGetLastError());
    }
    unsigned long long hs[2];
    PD_S_TRY(cudaMemcpyAsync(hs, scal, sizeof(hs), cudaMemcpyDeviceToHost, s));
    PD_S_TRY(cudaStreamSynchronize(s));
    if (exclusive_scan_i64(cf, frow, N, s) != PD_OK || exclusive_scan_i64(ca, arow, N, s) != PD_OK) {
        cleanup();
        return fail(PD_ERR_CUDA, "scan failed");
    }
    int64_t tot[2] = {0, 0};
    PD_S_TRY(cudaMemcpyAsync(&tot[0], frow + N, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    PD_S_TRY(cudaMemcpyAsync(&tot[1], arow + N, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    PD_S_TRY(cudaStreamSynchronize(s));
    PD_S_TRY(cudaMalloc(&fcol, sizeof(int32_t) * (tot[0] + 1)));
    PD_S_TRY(cudaMalloc(&fbr, sizeof(uint8_t) * (tot[0] + 1)));
    PD_S_TRY(cudaMalloc(&acol, sizeof(int32_t) * (tot[1] + 1)));
    const int cap = (int)hs[1] + 1;
    size_t sh = (size_t)wpb * cap * (sizeof(int32_t) + sizeof(uint8_t));
    if (sh > 200 * 1024) {
        cleanup();
        cudaFree(frow); cudaFree(arow); cudaFree(fcol); cudaFree(acol); cudaFree(fbr);
        return fail(PD_ERR_CAPACITY, "family larger than the search kernel's shared buffer");
    }
    if (sh > 48 * 1024)
        PD_S_TRY(cudaFuncSetAttribute(k_search<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh));
    if (N > 0) {
        k_search<1><<<blocks_for(N * 32, 32 * wpb), 32 * wpb, sh, s>>>(A, nullptr, nullptr, nullptr, nullptr, frow,
                                                                       fcol, fbr, arow, acol, cap);
        PD_S_TRY(cudaGetLastError());
    }
    PD_S_TRY(cudaStreamSynchronize(s));
#undef PD_S_TRY
    cleanup();
    *frow_o = frow;
    *fcol_o = fcol;
    *fbroken_o = fbr;
    *arow_o = arow;
    *acol_o = acol;
    *nh = tot[0];
    *nb = tot[0] - tot[1];
    *min_bond = __builtin_bit_cast(double, hs[0]);
    return PD_OK;
}

// ======================================= bond search without allocation

// pd_bond_search_noalloc works entirely in this fixed device array, carved
// into the regions below.  Every GPU that loads the library holds it until
// the process exits; all calls share it.
namespace na {
constexpr int64_t kNodes = PD_NOALLOC_MAX_NODES;
constexpr int64_t kCells = PD_NOALLOC_MAX_CELLS;
constexpr int kSlits = PD_NOALLOC_MAX_SLITS;
constexpr size_t kOffSorted = sizeof(int32_t) * kNodes;                 // node_cell [kNodes] at 0
constexpr size_t kOffCnt = kOffSorted + sizeof(int32_t) * kNodes;       // sorted [kNodes]
constexpr size_t kOffCellCnt = kOffCnt + sizeof(int64_t) * kNodes;      // cnt [kNodes]
constexpr size_t kOffCstart = kOffCellCnt + sizeof(int64_t) * (kCells + 1);
constexpr size_t kOffFill = kOffCstart + sizeof(int64_t) * (kCells + 1);
constexpr size_t kOffSlits = kOffFill + sizeof(int64_t) * (kCells + 1);
constexpr size_t kOffScal = kOffSlits + sizeof(double) * 6 * kSlits;   // bbox[6], min bits, max count
constexpr size_t kBytes = kOffScal + 16 * sizeof(double);
static_assert(kBytes == PD_NOALLOC_SCRATCH_BYTES, "scratch size stated in pdmtel_b200.h");
}  // namespace na

static __device__ __align__(256) unsigned char g_noalloc_scratch[na::kBytes];

namespace {

struct NaArgs {
    const double* x;  // [n][3], caller's device buffer
    int64_t n;
    double dx, delta, tol;
    SearchGrid g;
    unsigned char* s;  // device address of g_noalloc_scratch
    int nslit;
};

__device__ __forceinline__ int32_t* na_node_cell(unsigned char* s) { return (int32_t*)s; }
__device__ __forceinline__ int32_t* na_sorted(unsigned char* s) { return (int32_t*)(s + na::kOffSorted); }
__device__ __forceinline__ int64_t* na_cnt(unsigned char* s) { return (int64_t*)(s + na::kOffCnt); }
__device__ __forceinline__ int64_t* na_cell_cnt(unsigned char* s) { return (int64_t*)(s + na::kOffCellCnt); }
__device__ __forceinline__ int64_t* na_cstart(unsigned char* s) { return (int64_t*)(s + na::kOffCstart); }
__device__ __forceinline__ int64_t* na_fill(unsigned char* s) { return (int64_t*)(s + na::kOffFill); }
__device__ __forceinline__ double* na_slits(unsigned char* s) { return (double*)(s + na::kOffSlits); }
__device__ __forceinline__ double* na_scal(unsigned char* s) { return (double*)(s + na::kOffScal); }

// bounding box of the nodes into scal[0..5]; one block
__global__ void k_na_bbox(const double* __restrict__ x, int64_t n, unsigned char* s) {
    __shared__ double red[6][32];
    __shared__ int nonfinite;
    if (threadIdx.x == 0) nonfinite = 0;
    __syncthreads();
    double lo[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, hi[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
    bool bad = false;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x)
        for (int a = 0; a < 3; ++a) {
            bad = bad || !isfinite(x[3 * i + a]);
            lo[a] = dmin(lo[a], x[3 * i + a]);
            hi[a] = -dmin(-hi[a], -x[3 * i + a]);
        }
    if (bad) nonfinite = 1;
    for (int o = 16; o > 0; o >>= 1)
        for (int a = 0; a < 3; ++a) {
            lo[a] = dmin(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
            hi[a] = -dmin(-hi[a], -__shfl_xor_sync(0xffffffffu, hi[a], o));
        }
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0)
        for (int a = 0; a < 3; ++a) {
            red[a][w] = lo[a];
            red[3 + a][w] = hi[a];
        }
    __syncthreads();
    if (threadIdx.x == 0) {
        double* sc = na_scal(s);
        for (int a = 0; a < 3; ++a) {
            double l = red[a][0], h = red[3 + a][0];
            for (int k = 1; k < (int)(blockDim.x >> 5); ++k) {
                l = dmin(l, red[a][k]);
                h = -dmin(-h, -red[3 + a][k]);
            }
            sc[a] = nonfinite ? __longlong_as_double(0x7ff8000000000000LL) : l;  // a non-finite coordinate is reported as a NaN box
            sc[3 + a] = h;
        }
        ((unsigned long long*)sc)[6] = (unsigned long long)__double_as_longlong(0.0);
        ((unsigned long long*)sc)[7] = 0ull;
    }
}

__device__ __forceinline__ int64_t na_cell_of(const NaArgs& A, const double* p, int64_t* c) {
    for (int a = 0; a < 3; ++a) {
        int64_t v = (int64_t)floor((p[a] - A.g.lo[a]) / A.g.h);
        c[a] = v < 0 ? 0 : (v >= A.g.nc[a] ? A.g.nc[a] - 1 : v);
    }
    return (c[2] * A.g.nc[1] + c[1]) * A.g.nc[0] + c[0];
}

__global__ void k_na_cell_count(NaArgs A) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= A.n) return;
    int64_t c[3];
    const int64_t cell = na_cell_of(A, A.x + 3 * i, c);
    na_node_cell(A.s)[i] = (int32_t)cell;
    atomicAdd((unsigned long long*)&na_cell_cnt(A.s)[cell], 1ull);
}

// exclusive scan of in[0..n) into out[0..n], out[n] = total; one block of
// 1024 threads, each thread owning a contiguous run
__global__ void k_na_scan(const int64_t* __restrict__ in, int64_t* __restrict__ out, int64_t n) {
    __shared__ int64_t part[1024];
    const int64_t per = (n + 1023) / 1024;
    const int64_t b = threadIdx.x * per, e = b + per < n ? b + per : n;
    int64_t sum = 0;
    for (int64_t k = b; k < e; ++k) sum += in[k];
    part[threadIdx.x] = sum;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        const int64_t v = threadIdx.x >= o ? part[threadIdx.x - o] : 0;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    int64_t run = part[threadIdx.x] - sum;
    for (int64_t k = b; k < e; ++k) {
        const int64_t v = in[k];
        out[k] = run;
        run += v;
    }
    if (threadIdx.x == 1023) out[n] = part[1023];
}

__global__ void k_na_scatter(NaArgs A) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= A.n) return;
    const int32_t cell = na_node_cell(A.s)[i];
    const int64_t pos = (int64_t)atomicAdd((unsigned long long*)&na_fill(A.s)[cell], 1ull);
    na_sorted(A.s)[na_cstart(A.s)[cell] + pos] = (int32_t)i;
}

// One warp per node, the membership test of InitBond (pdDataManager2.cpp:
// 12-70).  PASS 0 counts; PASS 1 sorts the family by id in shared memory and
// writes it with the slit marks.
template <int PASS>
__global__ void k_na_search(NaArgs A, int64_t* row_ptr, int32_t* col, uint8_t* broken, int cap) {
    extern __shared__ int32_t sb[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    if (i >= A.n) return;
    int32_t* buf = sb + (size_t)wib * cap;
    uint8_t* brk = (uint8_t*)(sb + (size_t)(blockDim.x >> 5) * cap) + (size_t)wib * cap;
    const double* sl = na_slits(A.s);
    double pi[3] = {A.x[3 * i], A.x[3 * i + 1], A.x[3 * i + 2]};
    int64_t c[3];
    na_cell_of(A, pi, c);
    int64_t nf = 0;
    double mb = A.delta;
    for (int64_t dz = -1; dz <= 1; ++dz)
        for (int64_t dy = -1; dy <= 1; ++dy)
            for (int64_t dxc = -1; dxc <= 1; ++dxc) {
                const int64_t qx = c[0] + dxc, qy = c[1] + dy, qz = c[2] + dz;
                if (qx < 0 || qy < 0 || qz < 0 || qx >= A.g.nc[0] || qy >= A.g.nc[1] || qz >= A.g.nc[2]) continue;
                const int64_t q = (qz * A.g.nc[1] + qy) * A.g.nc[0] + qx;
                const int64_t s0 = na_cstart(A.s)[q], s1 = na_cstart(A.s)[q + 1];
                for (int64_t s = s0; s < s1; s += 32) {
                    bool hit = false, br = false;
                    int64_t j = -1;
                    if (s + lane < s1) {
                        j = na_sorted(A.s)[s + lane];
                        if (j != i) {
                            const double pj[3] = {A.x[3 * j], A.x[3 * j + 1], A.x[3 * j + 2]};
                            const double* pa = (i < j) ? pi : pj;
                            const double* pb = (i < j) ? pj : pi;
                            double dist;
                            hit = pair_bonded(pa, pb, A.dx, A.delta, A.tol, &dist);
                            if (hit) {
                                if (i < j) mb = dmin(mb, dist);
                                for (int k = 0; k < A.nslit; ++k) br = br || slit_crosses(sl + 6 * k, pa, pb);
                            }
                        }
                    }
                    const unsigned hm = __ballot_sync(0xffffffffu, hit);
                    if (PASS == 1 && hit) {
                        const int slot = (int)nf + __popc(hm & ((1u << lane) - 1u));
                        if (slot < cap) {
                            buf[slot] = (int32_t)j;
                            brk[slot] = br ? 1 : 0;
                        }
                    }
                    nf += __popc(hm);
                }
            }
    if (PASS == 0) {
        for (int o = 16; o > 0; o >>= 1) mb = dmin(mb, __shfl_xor_sync(0xffffffffu, mb, o));
        if (lane == 0) {
            na_cnt(A.s)[i] = nf;
            unsigned long long* sc = (unsigned long long*)na_scal(A.s);
            atomicMin(&sc[6], (unsigned long long)__double_as_longlong(mb));
            atomicMax(&sc[7], (unsigned long long)nf);
        }
        return;
    }
    __syncwarp();
    const int n = (int)(nf < cap ? nf : cap);
    const int64_t o = row_ptr[i];
    for (int e = lane; e < n; e += 32) {
        const int32_t v = buf[e];
        int rk = 0;
        for (int k = 0; k < n; ++k) rk += buf[k] < v ? 1 : 0;
        col[o + rk] = v;
        if (broken) broken[o + rk] = brk[e];
    }
}

std::mutex g_na_mu;
void* g_na_addr[64] = {};

}  // namespace

}  // namespace pd

extern "C" int pd_bond_search_noalloc(const double* coords, int64_t n, double grid_spacing, double horizon,
                                      int32_t num_slits, const double* slits, int64_t* row_ptr, int32_t* col,
                                      uint8_t* broken, int64_t capacity, void* stream, int64_t* num_halves,
                                      double* min_bond_length) {
    using namespace pd;
    if (n < 0 || n > na::kNodes) return fail(PD_ERR_CAPACITY, "pd_bond_search_noalloc: more nodes than PD_NOALLOC_MAX_NODES");
    if (num_slits < 0 || num_slits > na::kSlits || (num_slits > 0 && !slits))
        return fail(PD_ERR_ARG, "pd_bond_search_noalloc: bad slit list");
    if (!row_ptr || (n > 0 && !coords) || capacity < 0 || (capacity > 0 && !col) || !(grid_spacing > 0.0) ||
        !(horizon > 0.0))
        return fail(PD_ERR_ARG, "pd_bond_search_noalloc: bad argument");
    int dev = 0;
    PD_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(PD_ERR_ARG, "pd_bond_search_noalloc: device index above 63");
    unsigned char* s = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_na_mu);
        if (!g_na_addr[dev]) {
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess) return fail_cuda(e, "cudaGetSymbolAddress(g_noalloc_scratch)", __FILE__, __LINE__);
            g_na_addr[dev] = p;
        }
        s = (unsigned char*)g_na_addr[dev];
    }
    cudaStream_t st = (cudaStream_t)stream;
    double bb[6] = {0, 0, 0, 0, 0, 0};
    if (n > 0) {
        k_na_bbox<<<1, 1024, 0, st>>>(coords, n, s);
        PD_CUDA_TRY(cudaGetLastError());
        PD_CUDA_TRY(cudaMemcpyAsync(bb, s + na::kOffScal, sizeof bb, cudaMemcpyDeviceToHost, st));
        PD_CUDA_TRY(cudaStreamSynchronize(st));
    }
    NaArgs A;
    A.x = coords;
    A.n = n;
    A.dx = grid_spacing;
    A.delta = horizon;
    A.tol = 1.0e-4 * grid_spacing;
    A.s = s;
    A.nslit = num_slits;
    A.g.h = horizon + grid_spacing;
    // Cells per axis are counted in double and checked against the array's
    // limit before any conversion to an integer: a non-finite coordinate or a
    // horizon tiny next to the extent must not reach an undefined cast or an
    // overflowing product.
    int64_t ncell = 1;
    for (int a = 0; a < 3; ++a) {
        if (!std::isfinite(bb[a]) || !std::isfinite(bb[3 + a]))
            return fail(PD_ERR_ARG, "pd_bond_search_noalloc: non-finite coordinate");
        const double cells = std::floor((bb[3 + a] - bb[a]) / A.g.h) + 1.0;
        if (!(cells >= 1.0) || cells > (double)na::kCells)
            return fail(PD_ERR_CAPACITY, "pd_bond_search_noalloc: more cells than PD_NOALLOC_MAX_CELLS");
        A.g.lo[a] = bb[a];
        A.g.nc[a] = (int64_t)cells;
        ncell *= A.g.nc[a];  // each factor <= kCells and the partial product too: no overflow
        if (ncell > na::kCells)
            return fail(PD_ERR_CAPACITY, "pd_bond_search_noalloc: more cells than PD_NOALLOC_MAX_CELLS");
    }
    // the regions read before they are written start at zero
    PD_CUDA_TRY(cudaMemsetAsync(s + na::kOffCellCnt, 0, sizeof(int64_t) * (ncell + 1), st));
    PD_CUDA_TRY(cudaMemsetAsync(s + na::kOffFill, 0, sizeof(int64_t) * (ncell + 1), st));
    if (num_slits > 0)
        PD_CUDA_TRY(cudaMemcpyAsync(s + na::kOffSlits, slits, sizeof(double) * 6 * num_slits, cudaMemcpyHostToDevice, st));
    unsigned long long sc[2] = {(unsigned long long)__builtin_bit_cast(unsigned long long, horizon), 0ull};
    PD_CUDA_TRY(cudaMemcpyAsync(s + na::kOffScal + 6 * sizeof(double), sc, sizeof sc, cudaMemcpyHostToDevice, st));
    const int bs = 256, wpb = 4;
    const unsigned nb = (unsigned)((n + bs - 1) / bs), nw = (unsigned)((n * 32 + 32 * wpb - 1) / (32 * wpb));
    if (n > 0) k_na_cell_count<<<nb, bs, 0, st>>>(A);
    k_na_scan<<<1, 1024, 0, st>>>((const int64_t*)(s + na::kOffCellCnt), (int64_t*)(s + na::kOffCstart), ncell);
    if (n > 0) {
        k_na_scatter<<<nb, bs, 0, st>>>(A);
        k_na_search<0><<<nw, 32 * wpb, 0, st>>>(A, nullptr, nullptr, nullptr, 0);
    }
    k_na_scan<<<1, 1024, 0, st>>>((const int64_t*)(s + na::kOffCnt), row_ptr, n);
    PD_CUDA_TRY(cudaGetLastError());
    int64_t total = 0;
    unsigned long long back[2] = {0, 0};
    PD_CUDA_TRY(cudaMemcpyAsync(&total, row_ptr + n, sizeof total, cudaMemcpyDeviceToHost, st));
    PD_CUDA_TRY(cudaMemcpyAsync(back, s + na::kOffScal + 6 * sizeof(double), sizeof back, cudaMemcpyDeviceToHost, st));
    PD_CUDA_TRY(cudaStreamSynchronize(st));
    if (num_halves) *num_halves = total;
    if (min_bond_length) *min_bond_length = n > 0 ? __builtin_bit_cast(double, back[0]) : horizon;
    if (total > capacity) return fail(PD_ERR_CAPACITY, "pd_bond_search_noalloc: col capacity below the family size");
    const int cap = (int)back[1] + 1;
    const size_t sh = (size_t)wpb * cap * (sizeof(int32_t) + sizeof(uint8_t));
    if (sh > 48 * 1024) return fail(PD_ERR_CAPACITY, "pd_bond_search_noalloc: family larger than the shared buffer");
    if (n > 0) k_na_search<1><<<nw, 32 * wpb, sh, st>>>(A, row_ptr, col, broken, cap);
    PD_CUDA_TRY(cudaGetLastError());
    PD_CUDA_TRY(cudaStreamSynchronize(st));
    return PD_OK;
}

namespace pd {

// ================================================== areal force density
//
// pdSolve::PostAFD (pdSolve.cpp:810-834, pdDataManager3.cpp:442-635,
// 1101-1223): the stress tensor at a source node s from the areal force
// density.  For each direction d and each node i at s - (1 + is) dx e_d
// (is < int(horizon / dx)), the bond forces of i with every node j of its
// family that lies in the source's half space x_j,d >= x_s,d are summed.
// Here one thread takes one (i, s, d) item; the host builds the items and
// adds them up in the reference's order.

// Gauss-point displacements as PostAFD derives them from a Tecplot dump
// (pdDataManager.cpp:2704-2752, CalcApproxDispl, or the copy of the one-point
// rule): the MLS sum of the nodal displacements u_k c_k on every node, except
// that a direction a boundary condition flags keeps its Gauss points at zero
// (they are never set in a post-processing run).
__global__ void k_afd_gauss(Dev d, const double* __restrict__ U, double* __restrict__ ug) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= d.n) return;
    const int64_t N = d.n;
    const int npt = d.npt;
    bool flagged[3] = {false, false, false};
    if (d.bc[i] >= 0)
        for (int a = 0; a < 3; ++a) flagged[a] = d.bcs[d.bc[i]].dir[a] == 1;
    for (int g = 0; g < npt; ++g) {
        double v[3] = {0.0, 0.0, 0.0};
        if (d.mls) {
            const int64_t b = d.cbptr[i], nc = d.cbptr[i + 1] - b;
            for (int64_t k = 0; k < nc; ++k) {
                const int64_t m = d.cbidx[b + k];
                const double c = d.coeff[(b + k) * npt + g];
                v[0] += U[m] * c;
                v[1] += U[N + m] * c;
                v[2] += U[2 * N + m] * c;
            }
            for (int a = 0; a < 3; ++a)
                if (flagged[a]) v[a] = 0.0;
        } else {
            for (int a = 0; a < 3; ++a) v[a] = U[a * N + i];
        }
        for (int a = 0; a < 3; ++a) ug[(int64_t)(3 * g + a) * N + i] = v[a];
    }
}

// pdIntgManager::CalcBondBasedForce (pdIntgManager2.cpp:92-310), fixed
// Gauss points: the point at local position (X, Y, Z) from node i, with the
// displacement of cell j's point g
__device__ __forceinline__ void afd_point(const Dev& d, double X, double Y, double Z, const double* ugj, double ui0,
                                          double ui1, double ui2, double bE, double spring, double ecrit,
                                          double dxe, double* f) {
    const double xi1 = X - 0.0, xi2 = Y - 0.0, xi3 = Z - 0.0;
    const double eta1 = ugj[0] - ui0, eta2 = ugj[1] - ui1, eta3 = ugj[2] - ui2;
    const double r = sqrt(xi1 * xi1 + xi2 * xi2 + xi3 * xi3);
    const double y1 = xi1 + eta1, y2 = xi2 + eta2, y3 = xi3 + eta3;
    const double p = sqrt(y1 * y1 + y2 * y2 + y3 * y3);
    const double beta = beta_factor(r, d.delta, dxe, false);
    const double u = p - r;
    const double stretch = u / r;
    if (u <= 0.0 || (u > 0.0 && stretch <= ecrit)) {
        f[0] = bE * beta * spring * stretch * y1 / p;
        f[1] = bE * beta * spring * stretch * y2 / p;
        f[2] = bE * beta * spring * stretch * y3 / p;
    } else {
        f[0] = f[1] = f[2] = 0.0;
    }
}

__global__ void k_afd_items(Dev d, const double* __restrict__ U, const double* __restrict__ bE,
                            const double* __restrict__ ug, const double* __restrict__ absc,
                            const double* __restrict__ wts, int n1, int64_t n_items,
                            const int64_t* __restrict__ item_i, const int64_t* __restrict__ item_s,
                            const int32_t* __restrict__ item_d, double* __restrict__ out) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= n_items) return;
    const int64_t N = d.n;
    const int64_t i = item_i[t], s = item_s[t];
    const int dir = item_d[t] - 1;
    const double pi[3] = {d.x[i], d.x[N + i], d.x[2 * N + i]};
    const double xs_d = d.x[dir * N + s];
    const double ui0 = U[i], ui1 = U[N + i], ui2 = U[2 * N + i];
    const MatDev& Mi = d.mats[d.mat[i]];
    const double dx = d.dx, tol = 1.0e-4 * dx;
    double sum0 = 0.0, sum1 = 0.0, sum2 = 0.0;
    for (int64_t p = d.frow[i]; p < d.frow[i + 1]; ++p) {
        const int64_t j = d.fcol[p];
        const double pj[3] = {d.x[j], d.x[N + j], d.x[2 * N + j]};
        if (!(pj[dir] - xs_d >= 0.0)) continue;  // the source's R+ space
        const MatDev& Mj = d.mats[d.mat[j]];
        const double ecrit = dmin(Mi.ecrit, Mj.ecrit);
        const double spring = dmin(Mi.spring, Mj.spring);
        const double bEij = 0.5 * (bE[i] + bE[j]);
        double f[3] = {0.0, 0.0, 0.0};
        if (d.cci) {
            // pdDataManager::CalcBondForceCCI(bond, i, j), pdDataManager2.cpp:1087-1154
            const double xi1 = pj[0] - pi[0], xi2 = pj[1] - pi[1], xi3 = pj[2] - pi[2];
            const double eta1 = U[j] - ui0, eta2 = U[N + j] - ui1, eta3 = U[2 * N + j] - ui2;
            const double r = sqrt(xi1 * xi1 + xi2 * xi2 + xi3 * xi3);
            const double y1 = xi1 + eta1, y2 = xi2 + eta2, y3 = xi3 + eta3;
            const double pl = sqrt(y1 * y1 + y2 * y2 + y3 * y3);
            const double u = pl - r;
            const double stretch = u / r;
            if (u <= 0.0 || (u > 0.0 && stretch <= ecrit)) {
                const double beta = beta_factor(r, d.delta, dx, !d.cci_mdf);
                const double vol = d.vol;
                f[0] = bEij * vol * beta * spring * stretch * y1 / pl;
                f[1] = bEij * vol * beta * spring * stretch * y2 / pl;
                f[2] = bEij * vol * beta * spring * stretch * y3 / pl;
            }
        } else {
            // CalcBondForceIntg (pdDataManager2.cpp:1156-1215): nothing when
            // the cell lies beyond the horizon, else the cell's fixed Gauss
            // rule as pdIntgManager::CalcConfigurationType3 / CalcIntg3D /
            // CalcGaussianQuad nest it (pdIntgManager.cpp:49-128,453-509,
            // 3471-3482), in local coordinates x_j - x_i
            double mn = kMega, a, b;
            for (int ax = 0; ax < 3; ++ax) {
                dist_to_face(ax + 1, pj[ax] - 0.5 * dx, pi, pj, dx, &a, &b);
                mn = dmin(mn, a);
                dist_to_face(ax + 1, pj[ax] + 0.5 * dx, pi, pj, dx, &a, &b);
                mn = dmin(mn, a);
            }
            if (!(d.delta <= mn)) {
                const double x1j = pj[0] - pi[0], x2j = pj[1] - pi[1], x3j = pj[2] - pi[2];
                const double lo1 = x1j - 0.5 * dx, hi1 = x1j + 0.5 * dx;
                const double lo2 = x2j - 0.5 * dx, hi2 = x2j + 0.5 * dx;
                const double lo3 = x3j - 0.5 * dx, hi3 = x3j + 0.5 * dx;
                int counter = 0;  // _intgPointCounter: the Gauss point of cell j
                if (fabs(lo1 - hi1) > 1.0e-10) {
                    double S1[3] = {0.0, 0.0, 0.0};
                    for (int q1 = 0; q1 < n1; ++q1) {
                        const double X = 0.5 * dx * absc[q1] + x1j;
                        double F2[3] = {0.0, 0.0, 0.0};
                        if (fabs(lo2 - hi2) > 1.0e-10) {
                            double S2[3] = {0.0, 0.0, 0.0};
                            for (int q2 = 0; q2 < n1; ++q2) {
                                const double Y = 0.5 * dx * absc[q2] + x2j;
                                double F3[3] = {0.0, 0.0, 0.0};
                                if (fabs(lo3 - hi3) > 1.0e-10) {
                                    double S3[3] = {0.0, 0.0, 0.0};
                                    for (int q3 = 0; q3 < n1; ++q3) {
                                        const double Z = 0.5 * dx * absc[q3] + x3j;
                                        const double ugj[3] = {ug[(int64_t)(3 * counter) * N + j],
                                                               ug[(int64_t)(3 * counter + 1) * N + j],
                                                               ug[(int64_t)(3 * counter + 2) * N + j]};
                                        double fp[3];
                                        afd_point(d, X, Y, Z, ugj, ui0, ui1, ui2, bEij, spring, ecrit,
                                                  d.gc[counter].dxe, fp);
                                        ++counter;
                                        for (int c = 0; c < 3; ++c) S3[c] += wts[q3] * fp[c];
                                    }
                                    for (int c = 0; c < 3; ++c) F3[c] = S3[c] * (0.5 * (hi3 - lo3));
                                }
                                for (int c = 0; c < 3; ++c) S2[c] += wts[q2] * F3[c];
                            }
                            for (int c = 0; c < 3; ++c) F2[c] = S2[c] * (0.5 * (hi2 - lo2));
                        }
                        for (int c = 0; c < 3; ++c) S1[c] += wts[q1] * F2[c];
                    }
                    for (int c = 0; c < 3; ++c) f[c] = S1[c] * (0.5 * (hi1 - lo1));
                }
            }
        }
        sum0 += f[0];
        sum1 += f[1];
        sum2 += f[2];
    }
    (void)tol;
    out[3 * t] = sum0;
    out[3 * t + 1] = sum1;
    out[3 * t + 2] = sum2;
}

int afd_forces(const Dev& d, const double* U, const double* bE, double* ug, const double* absc, const double* wts,
               int n1, int64_t n_items, const int64_t* item_i, const int64_t* item_s, const int32_t* item_d,
               double* out, cudaStream_t s) {
    if (d.n == 0 || n_items == 0) return PD_OK;
    k_afd_gauss<<<(unsigned)((d.n + 127) / 128), 128, 0, s>>>(d, U, ug);
    k_afd_items<<<(unsigned)((n_items + 63) / 64), 64, 0, s>>>(d, U, bE, ug, absc, wts, n1, n_items, item_i, item_s,
                                                               item_d, out);
    return cudaGetLastError() == cudaSuccess ? PD_OK : PD_ERR_CUDA;
}

}  // namespace pd
