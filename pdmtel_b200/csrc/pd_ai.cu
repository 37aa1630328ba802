// Adaptive-trapezoid (AI) form on the device: the ai_on branch of
// CalcBondBasedMotionRK4 (pdDataManager.cpp:1886-1915) with
// CalcBondForceIntg (pdDataManager2.cpp:1227-1291) and the integrand
// pdIntgManager::CalcBondBasedForce (pdIntgManager2.cpp:92-310).
//
// Compiled with -fmad=false: the nested trapezoid sums (pd_ai_eval.h), the
// MLS sums and the force are rounded operation by operation in the
// reference's order, so the stage's velocity buffer is the reference's bit
// for bit.
//
// One stage is three launches:
//  k_ai_gather  one thread per MLS table entry: the displacement of the
//               entry's point from the trial displacements (the reference
//               forms it point by point inside the integrand; the sum is the
//               same, so it is formed once per entry here and read by every
//               bond to the node);
//  k_ai_bond    one warp per full-family entry i -> j: the bond's force and
//               the count of its points past the critical stretch; with the
//               energy on, every point's energy term in the bond's slots of a
//               per-point buffer (0.0 for a failed point);
//  k_ai_sum     one thread per node (one warp with the energy on,
//               k_ai_sum_energy): the velocity update bond by bond in family
//               order, and the energy terms added point by point in the
//               reference's order (a sequential sum, formed exactly).
//               A failing point breaks the bond object the two
//               nodes share (pdIntgManager2.cpp:301-308), and the reference
//               visits node i's bonds after those of every lower node: a bond
//               to a lower node j is skipped when j's evaluation of it failed
//               in this stage.  Breaks are committed here for the next stage.
#include <cfloat>
#include <cmath>

#include "pd_ai_eval.h"
#include "pd_internal.cuh"
#include "pd_stage.cuh"

namespace pd {

namespace {

__device__ __forceinline__ double dmin(double a, double b) { return (b < a) ? b : a; }  // std::min

__global__ void k_ai_gather(Dev d, const double* __restrict__ us) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= d.ai_ntab) return;
    const int64_t N = d.n;
    const int64_t j = d.ai_tnode[e];
    const int64_t k = e - d.ai_tptr[j];
    const int64_t c0 = d.cbptr[j], nc = d.cbptr[j + 1] - c0;
    const double* cf = d.ai_tcoef + d.ai_coff[j] + k * nc;
    const int32_t* cb = d.cbidx + c0;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    for (int64_t q = 0; q < nc; ++q) {
        const int64_t m = cb[q];
        const double c = cf[q];
        a0 += us[m] * c;
        a1 += us[N + m] * c;
        a2 += us[2 * N + m] * c;
    }
    d.ai_u[3 * e] = a0;
    d.ai_u[3 * e + 1] = a1;
    d.ai_u[3 * e + 2] = a2;
}

// The integrand at one trapezoid point of bond i -> j: the force density into
// f, the energy term into *e (0.0 for a point past the critical stretch);
// returns 1 for such a point.  k: the point's index in its region (the entry
// of node j's MLS list the reference reads).
struct ForceFn {
    const Dev* d;
    double ui[3];
    double xi[3];        // node i (global): a DISPLGRAD point sits at local + x_i
    double ecrit, c, be;
    const double* tab;   // node j's table entries [K][3]
    int64_t K;
    const BcDev* B;      // node j's boundary condition or null
    double fac;

    __device__ int eval(const double* p, int k, double* f, double* e) const {
        double eta[3];
        if (d->ai_mls) {
            double u[3];
            if (k < K) {
                u[0] = tab[3 * k];
                u[1] = tab[3 * k + 1];
                u[2] = tab[3 * k + 2];
            } else {
                u[0] = u[1] = u[2] = 0.0;
                *d->ai_err = 1;
            }
            if (B) {
                for (int a = 0; a < 3; ++a) {
                    if (B->dir[a] != 1) continue;
                    if (B->type == PD_BC_DISPL) {
                        u[a] = B->val[a] * fac;
                    } else if (B->type == PD_BC_DISPLGRAD) {
                        const double g0 = p[0] + xi[0], g1 = p[1] + xi[1], g2 = p[2] + xi[2];
                        u[a] = (B->val[3 * a] * g0 + B->val[3 * a + 1] * g1 + B->val[3 * a + 2] * g2) * fac;
                    }
                }
            }
            eta[0] = u[0] - ui[0];
            eta[1] = u[1] - ui[1];
            eta[2] = u[2] - ui[2];
        } else {
            // every family node carries a displacement gradient (checked at upload)
            for (int a = 0; a < 3; ++a)
                eta[a] = B->val[3 * a] * (p[0] - 0.0) + B->val[3 * a + 1] * (p[1] - 0.0) +
                         B->val[3 * a + 2] * (p[2] - 0.0);
        }
        const double x0 = p[0] - 0.0, x1 = p[1] - 0.0, x2 = p[2] - 0.0;
        const double r = sqrt(x0 * x0 + x1 * x1 + x2 * x2);
        const double y0 = x0 + eta[0], y1 = x1 + eta[1], y2 = x2 + eta[2];
        const double pl = sqrt(y0 * y0 + y1 * y1 + y2 * y2);
        const double u = pl - r;
        const double s = u / r;
        if (u <= 0.0 || (u > 0.0 && s <= ecrit)) {
            const double t = be * 1.0 * c * s;
            f[0] = t * y0 / pl;
            f[1] = t * y1 / pl;
            f[2] = t * y2 / pl;
            *e = be * 0.5 * (0.5 * 1.0 * (c / r) * u * u);
            return 0;
        }
        f[0] = f[1] = f[2] = 0.0;
        *e = 0.0;
        return 1;
    }
};

__device__ __forceinline__ void node_u(const Dev& d, int64_t i, double* u) {
    const int64_t N = d.n;
    const double* src = d.bc[i] >= 0 ? d.U : d.us;
    u[0] = src[i];
    u[1] = src[N + i];
    u[2] = src[2 * N + i];
}

constexpr int kAiWarps = 4;  // warps per block of k_ai_bond

// One warp per bond, region by region.  Lane r < np^2 owns row r = (k, l) of
// the region (outer point k, middle point l): its limits, whether its inner
// interval is empty, and by a warp prefix sum the region index of its first
// point.  The np^3 points are then spread over the lanes, each point's
// integrand written to shared memory; the row, middle and outer trapezoid
// sums follow in the order of pdIntgManager::CalcTrapzdQuad (lane = row,
// lane = outer point, lane 0), so the integral is the serial one bit for bit.
template <bool ENERGY>
__global__ void __launch_bounds__(128) k_ai_bond(Dev d) {
    using namespace pd_ai;
    constexpr unsigned full = 0xffffffffu;
    __shared__ double sf[kAiWarps][kMaxRegionPoints][3];
    __shared__ double sh[kAiWarps][kMaxPerDir * kMaxPerDir][3];
    __shared__ double sg[kAiWarps][kMaxPerDir][3];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    if (w >= d.ai_nent) return;
    const int64_t p = d.ai_order[w];
    if (d.ai_brk[p]) {
        if (lane == 0) d.ai_fail[p] = 0;
        if (ENERGY)  // no terms: the node's sum streams over these slots
            for (int64_t e = d.ai_eptr[p] + lane; e < d.ai_eptr[p + 1]; e += 32) d.ai_e[e] = 0.0;
        return;
    }
    const int64_t N = d.n;
    const int64_t i = d.ai_row[p], j = d.fcol[p];
    const double t_now = *d.tdev;
    ForceFn fn;
    fn.d = &d;
    node_u(d, i, fn.ui);
    fn.xi[0] = d.x[i];
    fn.xi[1] = d.x[N + i];
    fn.xi[2] = d.x[2 * N + i];
    const MatDev& Mi = d.mats[d.mat[i]];
    const MatDev& Mj = d.mats[d.mat[j]];
    fn.ecrit = dmin(Mi.ecrit, Mj.ecrit);
    fn.c = dmin(Mi.spring, Mj.spring);
    if (d.sfac) fn.c = fn.c * (0.5 * (d.sfac[i] + d.sfac[j]));
    fn.be = 0.5 * (d.bdry[i] + d.bdry[j]);
    const int b = d.bc[j];
    fn.B = b >= 0 ? &d.bcs[b] : nullptr;
    fn.fac = b >= 0 ? bc_time_factor(d.bcs[b], t_now) : 0.0;
    fn.tab = d.ai_mls ? d.ai_u + 3 * d.ai_tptr[j] : nullptr;
    fn.K = d.ai_mls ? d.ai_tptr[j + 1] - d.ai_tptr[j] : 0;
    const double xj[3] = {d.x[j] - d.x[i], d.x[N + j] - d.x[N + i], d.x[2 * N + j] - d.x[2 * N + i]};
    const double delta = d.delta, dx = d.dx;
    const int n = d.ai_n, np = points_per_dir(n), nrow = np * np;
    double F[3] = {0.0, 0.0, 0.0};
    int fail = 0;
    int64_t q0 = ENERGY ? d.ai_eptr[p] : 0;
    const int64_t r0 = d.ai_rptr[p], r1 = d.ai_rptr[p + 1];
    const bool assign = r1 > r0 && (d.ai_reg[r0].flags & PD_AI_ASSIGN);
    for (int64_t r = r0; r < r1; ++r) {
        const pd_ai_region R = d.ai_reg[r];
        double out[3] = {0.0, 0.0, 0.0};
        if (!(fabs(R.a - R.b) <= 1.0e-10)) {
            // rows
            double t = 0.0, s = 0.0, ml = 0.0, mh = 0.0, zl = 0.0, zh = 0.0;
            int mid_ok = 0, row_ok = 0;
            if (lane < nrow) {
                t = point(n, lane / np, R.a, R.b);
                ml = mid_limit(R.lim[0], t, xj, delta, dx);
                mh = mid_limit(R.lim[1], t, xj, delta, dx);
                mid_ok = !(fabs(ml - mh) <= 1.0e-10);
                if (mid_ok) {
                    s = point(n, lane % np, ml, mh);
                    zl = in_limit(R.lim[2], t, s, xj, delta, dx);
                    zh = in_limit(R.lim[3], t, s, xj, delta, dx);
                    row_ok = !(fabs(zl - zh) <= 1.0e-10);
                }
            }
            const int cnt = row_ok ? np : 0;
            int incl = cnt;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const int v = __shfl_up_sync(full, incl, off);
                if (lane >= off) incl += v;
            }
            const int base = incl - cnt;
            const int total = __shfl_sync(full, incl, 31);
            // points
            const int nslot = nrow * np;
            for (int s0 = 0; s0 < nslot; s0 += 32) {
                const int slot = s0 + lane;
                const int row = slot < nslot ? slot / np : 0;
                const double rt = __shfl_sync(full, t, row), rs = __shfl_sync(full, s, row);
                const double rzl = __shfl_sync(full, zl, row), rzh = __shfl_sync(full, zh, row);
                const int rok = __shfl_sync(full, row_ok, row), rbase = __shfl_sync(full, base, row);
                if (slot < nslot && rok) {
                    const int m = slot - row * np;
                    double pp[3], f[3], e;
                    pp[R.axis[0]] = rt;
                    pp[R.axis[1]] = rs;
                    pp[R.axis[2]] = point(n, m, rzl, rzh);
                    fail += fn.eval(pp, rbase + m, f, &e);
                    sf[wib][slot][0] = f[0];
                    sf[wib][slot][1] = f[1];
                    sf[wib][slot][2] = f[2];
                    if (ENERGY) d.ai_e[q0 + rbase + m] = e;
                }
            }
            __syncwarp();
            // inner sums, one lane per row
            if (lane < nrow) {
                double h[3] = {0.0, 0.0, 0.0};
                if (row_ok) {
                    double acc[3];
                    for (int m = 0; m < np; ++m) accumulate(m, np, sf[wib][lane * np + m], acc);
                    const double wgt = scale(n, zl, zh);
                    h[0] = wgt * acc[0];
                    h[1] = wgt * acc[1];
                    h[2] = wgt * acc[2];
                }
                sh[wib][lane][0] = h[0];
                sh[wib][lane][1] = h[1];
                sh[wib][lane][2] = h[2];
            }
            __syncwarp();
            // middle sums, one lane per outer point (row k np holds its limits)
            const int src = lane < np ? lane * np : 0;
            const double kml = __shfl_sync(full, ml, src), kmh = __shfl_sync(full, mh, src);
            const int kok = __shfl_sync(full, mid_ok, src);
            if (lane < np) {
                double g[3] = {0.0, 0.0, 0.0};
                if (kok) {
                    double acc[3];
                    for (int l = 0; l < np; ++l) accumulate(l, np, sh[wib][lane * np + l], acc);
                    const double wgt = scale(n, kml, kmh);
                    g[0] = wgt * acc[0];
                    g[1] = wgt * acc[1];
                    g[2] = wgt * acc[2];
                }
                sg[wib][lane][0] = g[0];
                sg[wib][lane][1] = g[1];
                sg[wib][lane][2] = g[2];
            }
            __syncwarp();
            if (lane == 0) {
                double acc[3];
                for (int k = 0; k < np; ++k) accumulate(k, np, sg[wib][k], acc);
                const double wgt = scale(n, R.a, R.b);
                out[0] = wgt * acc[0];
                out[1] = wgt * acc[1];
                out[2] = wgt * acc[2];
            }
            __syncwarp();
            q0 += total;
        }
        if (assign) {
            F[0] = out[0];
            F[1] = out[1];
            F[2] = out[2];
        } else {
            F[0] = F[0] + out[0];
            F[1] = F[1] + out[1];
            F[2] = F[2] + out[2];
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) fail += __shfl_down_sync(full, fail, off);
    if (lane == 0) {
        d.ai_F[3 * p] = F[0];
        d.ai_F[3 * p + 1] = F[1];
        d.ai_F[3 * p + 2] = F[2];
        d.ai_fail[p] = fail;
    }
}

__global__ void k_ai_sum(Dev d, double dts) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= d.n) return;
    const int64_t N = d.n;
    const MatDev Mi = d.mats[d.mat[i]];
    const double rho = Mi.density;
    const double b0 = Mi.grav[0] * rho, b1 = Mi.grav[1] * rho, b2 = Mi.grav[2] * rho;
    double v0 = d.vbuf[i], v1 = d.vbuf[N + i], v2 = d.vbuf[2 * N + i];
    int dmg = d.ai_dmg[i];
    const int64_t pe = d.frow[i + 1];
    for (int64_t p = d.frow[i]; p < pe; ++p) {
        if (d.ai_brk[p]) continue;
        const int64_t j = d.fcol[p];
        const int64_t q = d.ai_mirror[p];
        if (j < i && d.ai_fail[q] > 0) {
            d.ai_brk[p] = 1;  // broken by node j's visit of this bond in this stage
            continue;
        }
        const double F[3] = {d.ai_F[3 * p], d.ai_F[3 * p + 1], d.ai_F[3 * p + 2]};
        dmg += d.ai_fail[p];
        v0 += (F[0] + b0) * dts / rho;
        v1 += (F[1] + b1) * dts / rho;
        v2 += (F[2] + b2) * dts / rho;
        if (d.ai_fail[p] > 0 || (j > i && d.ai_fail[q] > 0)) d.ai_brk[p] = 1;
    }
    d.vbuf[i] = v0;
    d.vbuf[N + i] = v1;
    d.vbuf[2 * N + i] = v2;
    d.ai_dmg[i] = dmg;
}

// With the energy on: one warp per node.  The node's energy terms are
// contiguous (its entries' slots in family order; k_ai_bond zeroes the slots
// of bonds broken before the stage, and adding +0.0 to a non-negative sum
// changes nothing), so the warp streams them 128 at a time through shared
// memory, the next round's loads in flight while lane 0 adds the current
// round in point order: the reference's sequential sum, formed exactly.  A
// node with a bond its lower node broke in this stage (rare) takes the terms
// bond by bond instead.  Lane 0 then does the velocity update and the break
// bookkeeping of k_ai_sum.
__global__ void __launch_bounds__(128) k_ai_sum_energy(Dev d, double dts) {
    constexpr int kRound = 128;
    __shared__ double buf[4][2][kRound];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    if (i >= d.n) return;
    const int64_t N = d.n;
    const int64_t pb = d.frow[i], pe = d.frow[i + 1];
    // a bond skipped because node j's visit of it failed in this stage?
    int skip = 0;
    for (int64_t p = pb + lane; p < pe; p += 32) {
        const int64_t j = d.fcol[p];
        if (!d.ai_brk[p] && j < i && d.ai_fail[d.ai_mirror[p]] > 0) skip = 1;
    }
    skip = __any_sync(0xffffffffu, skip);
    double eacc = d.eed[i];
    auto stream = [&](int64_t E0, int64_t E1) {
        double nxt[kRound / 32];
#pragma unroll
        for (int u = 0; u < kRound / 32; ++u) {
            const int64_t e = E0 + 32 * u + lane;
            nxt[u] = e < E1 ? d.ai_e[e] : 0.0;
        }
        int cur = 0;
        for (int64_t base = E0; base < E1; base += kRound) {
#pragma unroll
            for (int u = 0; u < kRound / 32; ++u) buf[wib][cur][32 * u + lane] = nxt[u];
            __syncwarp();
#pragma unroll
            for (int u = 0; u < kRound / 32; ++u) {
                const int64_t e = base + kRound + 32 * u + lane;
                nxt[u] = e < E1 ? d.ai_e[e] : 0.0;
            }
            if (lane == 0) {
                const int m = (E1 - base) < kRound ? (int)(E1 - base) : kRound;
                const double* b = buf[wib][cur];
                int k = 0;
                // eight shared-memory loads in flight ahead of the in-order adds
                for (; k + 8 <= m; k += 8) {
                    double v[8];
#pragma unroll
                    for (int u = 0; u < 8; ++u) v[u] = b[k + u];
#pragma unroll
                    for (int u = 0; u < 8; ++u) eacc += v[u];
                }
                for (; k < m; ++k) eacc += b[k];
            }
            cur ^= 1;
        }
        __syncwarp();
    };
    if (!skip) {
        stream(d.ai_eptr[pb], d.ai_eptr[pe]);
    } else {
        for (int64_t p = pb; p < pe; ++p) {
            if (d.ai_brk[p]) continue;
            const int64_t j = d.fcol[p];
            if (j < i && d.ai_fail[d.ai_mirror[p]] > 0) continue;
            stream(d.ai_eptr[p], d.ai_eptr[p + 1]);
        }
    }
    if (lane != 0) return;
    const MatDev Mi = d.mats[d.mat[i]];
    const double rho = Mi.density;
    const double b0 = Mi.grav[0] * rho, b1 = Mi.grav[1] * rho, b2 = Mi.grav[2] * rho;
    double v0 = d.vbuf[i], v1 = d.vbuf[N + i], v2 = d.vbuf[2 * N + i];
    int dmg = d.ai_dmg[i];
    for (int64_t p = pb; p < pe; ++p) {
        if (d.ai_brk[p]) continue;
        const int64_t j = d.fcol[p];
        const int64_t q = d.ai_mirror[p];
        if (j < i && d.ai_fail[q] > 0) {
            d.ai_brk[p] = 1;  // broken by node j's visit of this bond in this stage
            continue;
        }
        dmg += d.ai_fail[p];
        v0 += (d.ai_F[3 * p] + b0) * dts / rho;
        v1 += (d.ai_F[3 * p + 1] + b1) * dts / rho;
        v2 += (d.ai_F[3 * p + 2] + b2) * dts / rho;
        if (d.ai_fail[p] > 0 || (j > i && d.ai_fail[q] > 0)) d.ai_brk[p] = 1;
    }
    d.vbuf[i] = v0;
    d.vbuf[N + i] = v1;
    d.vbuf[2 * N + i] = v2;
    d.ai_dmg[i] = dmg;
    d.eed[i] = eacc;
}

inline unsigned blocks_for(int64_t n, int bs) { return (unsigned)((n + bs - 1) / bs); }

}  // namespace

void launch_ai_gather(const Dev& d, const double* us, cudaStream_t s) {
    if (!d.ai_mls || d.ai_ntab == 0) return;
    k_ai_gather<<<blocks_for(d.ai_ntab, 256), 256, 0, s>>>(d, us);
}

void launch_ai_force(const Dev& d, double dts, cudaStream_t s) {
    if (d.n == 0) return;
    if (d.ai_nent > 0) {
        const unsigned nb = blocks_for(d.ai_nent, kAiWarps);
        if (d.energy) k_ai_bond<true><<<nb, 32 * kAiWarps, 0, s>>>(d);
        else k_ai_bond<false><<<nb, 32 * kAiWarps, 0, s>>>(d);
    }
    if (d.energy) k_ai_sum_energy<<<blocks_for(32 * d.n, 128), 128, 0, s>>>(d, dts);
    else k_ai_sum<<<blocks_for(d.n, 128), 128, 0, s>>>(d, dts);
}

}  // namespace pd
