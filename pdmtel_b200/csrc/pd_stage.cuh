// The per-node end of an RK4 stage, shared by the stage kernel of every form
// and by the persistent kernel.
//
// Every operation is an explicit round-to-nearest intrinsic, in the order the
// reference writes it, so the result is the same bit for bit whatever the
// contraction flags of the translation unit that includes this file.  Loads
// of the state go through L2 (ld.global.cg): inside one persistent launch
// another SM may have rewritten a line this SM still holds in L1.
#pragma once

#include "pd_internal.cuh"

namespace pd {

// GetTimeFactor: VELOC is on until its end time; DISPL/DISPLGRAD ramp as
// t/t_end when load_type == 1, else full (pdDataManager.cpp:2507-2522)
__device__ __forceinline__ double bc_time_factor(const BcDev& b, double t) {
    if (b.type == PD_BC_VELOC) return (t <= b.end_time) ? 1.0 : 0.0;
    if (b.load_type == 1.0) return (t <= b.end_time) ? __ddiv_rn(t, b.end_time) : 1.0;
    return 1.0;
}

// After the bond forces of stage `stage` (1..4; 0 for a lone stage whose k
// goes to k1) have been added to vbuf at time t: the traction load (project
// rule: value*factor/dx added to vbuf once per stage), UpdateNodeStatusWithBC
// (pdDataManager.cpp:2497-2602), k = vbuf*dt_s (:1977-1990) and the RK4
// bookkeeping of pdDataManager::RK4 (:2027-2092).  With ENERGY, stage 4
// leaves the node's kinetic and elastic energy in red[i], red[N+i].
template <bool ENERGY>
__device__ __forceinline__ void stage_epilogue(const Dev& d, int64_t i, int stage, double dts, double dt, double t) {
    const int64_t N = d.n;
    const double rho = d.mats[d.mat[i]].density;
    double v[3] = {__ldcg(d.vbuf + i), __ldcg(d.vbuf + N + i), __ldcg(d.vbuf + 2 * N + i)};
    double U[3] = {__ldcg(d.U + i), __ldcg(d.U + N + i), __ldcg(d.U + 2 * N + i)};
    const int b = d.bc[i];
    if (b >= 0) {
        const BcDev& B = d.bcs[b];
        const double fac = bc_time_factor(B, t);
        const double X[3] = {d.x[i], d.x[N + i], d.x[2 * N + i]};
        for (int a = 0; a < 3; ++a) {
            if (B.dir[a] != 1) continue;
            if (B.type == PD_BC_TRACTION) {
                const double tb = __ddiv_rn(__dmul_rn(B.val[a], fac), d.dx);
                v[a] = __dadd_rn(v[a], __ddiv_rn(__dmul_rn(tb, dts), rho));
            } else if (B.type == PD_BC_DISPL) {
                U[a] = __dmul_rn(B.val[a], fac);
                v[a] = 0.0;
            } else if (B.type == PD_BC_VELOC) {
                v[a] = __dmul_rn(B.val[a], fac);
            } else if (B.type == PD_BC_DISPLGRAD) {
                const double e = __dadd_rn(__dadd_rn(__dmul_rn(B.val[3 * a], X[0]), __dmul_rn(B.val[3 * a + 1], X[1])),
                                           __dmul_rn(B.val[3 * a + 2], X[2]));
                U[a] = __dmul_rn(e, fac);
                v[a] = 0.0;
            }
        }
    }
    const double dt6 = 1.0 / 6.0;
    for (int a = 0; a < 3; ++a) {
        const int64_t r = a * N + i;
        const double k = __dmul_rn(v[a], dts);
        if (stage == 0) {
            d.k1[r] = k;
        } else if (stage == 1) {
            d.k1[r] = k;
            d.us[r] = __dadd_rn(__ldcg(d.u1 + r), __dmul_rn(0.5, k));
        } else if (stage == 2) {
            d.k2[r] = k;
            d.us[r] = __dadd_rn(__ldcg(d.u1 + r), __dmul_rn(0.5, k));
        } else if (stage == 3) {
            d.us[r] = __dadd_rn(__ldcg(d.u1 + r), k);
            d.k32[r] = __dadd_rn(k, __ldcg(d.k2 + r));
        } else {
            const double Vold = __ldcg(d.V + r);
            const double inc =
                __dmul_rn(dt6, __dadd_rn(__dadd_rn(__ldcg(d.k1 + r), k), __dmul_rn(2.0, __ldcg(d.k32 + r))));
            if (b >= 0) {
                U[a] = __dadd_rn(U[a], inc);
            } else {
                const double damp = __ddiv_rn(__dmul_rn(__dmul_rn(__dmul_rn(dt, d.damping), Vold), dt), rho);
                U[a] = __dsub_rn(__dadd_rn(U[a], inc), damp);
            }
            v[a] = __dadd_rn(v[a], __ddiv_rn(__dmul_rn(__dmul_rn(-d.damping, Vold), dt), rho));
            d.V[r] = v[a];
            d.u1[r] = U[a];
            d.us[r] = U[a];
        }
        d.vbuf[r] = v[a];
        d.U[r] = U[a];
    }
    if (ENERGY && stage == 4) {
        const double velsq = __dadd_rn(__dadd_rn(__dmul_rn(v[0], v[0]), __dmul_rn(v[1], v[1])), __dmul_rn(v[2], v[2]));
        d.red[i] = __dmul_rn(__dmul_rn(__dmul_rn(0.5, rho), velsq), d.vol);
        d.red[N + i] = __dmul_rn(d.vol, __ldcg(d.eed + i));
    }
}

}  // namespace pd
