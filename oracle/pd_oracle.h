/*
 * pd_oracle — CPU restatement of the pdMTEL hot path, used ONLY as a checker.
 *
 * This is test infrastructure.  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg load it; the product library never links it.
 *
 * Every function restates the reference's arithmetic in the reference's own
 * operation order, so that (compiled with -ffp-contract=off, as the reference
 * build is) it reproduces the reference bit for bit.  Parity of this
 * restatement is pinned against the reference itself (oracle/ref_harness.cpp
 * dumps, committed under tests/golden/).  The parts the reference does not
 * implement — slit deletion, the traction load, the per-node micromodulus
 * factor and the static operator's solver — follow the project rules stated at
 * each function and are "parity unpinned" by the reference.
 */
#ifndef PD_ORACLE_H
#define PD_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* boundary-condition types, pdDataManager.h:231 */
enum { OR_DISPL = 1, OR_VELOC = 2, OR_DISPLGRAD = 3, OR_TRACTION = 4 };

typedef struct or_model {
    int64_t n;                 /* nodes */
    const double* x;           /* [n][3] reference coordinates */
    double dx, delta;          /* grid spacing, horizon */
    int cci, cci_mdf;          /* CCI flags (pdDataManager.cpp:597-610) */
    int mls;                   /* MLS on (FGI with n>1) */
    int npt;                   /* Gauss points per node (n^3) */
    const double* xg;          /* [n][npt][3] Gauss point coordinates */
    const double* gw;          /* [npt][3] Gauss weights per axis */
    const int64_t* fam_ptr;    /* [n+1] family CSR, ascending ids */
    const int32_t* fam_col;
    const uint8_t* broken;     /* [H] per family entry */
    const int64_t* cb_ptr;     /* [n+1] MLS contributors (NULL if !mls) */
    const int32_t* cb_idx;
    const double* coeff;       /* per node: npt blocks of ncb coefficients */
    const double* bdry_eff;    /* [n] */
    const int32_t* mat;        /* [n] material index */
    const double* mat_spring;  /* per material */
    const double* mat_ecrit;
    const double* mat_density;
    const double* mat_grav;    /* [nmat][3] */
    const double* mat_ymod;
    const int32_t* bc;         /* [n] bc index or -1 */
    const int32_t* bc_type;    /* per bc */
    const int32_t* bc_dir;     /* [nbc][3] */
    const double* bc_val;      /* [nbc][9] */
    const double* bc_end;
    const double* bc_load;
    const double* spring_factor; /* [n] per-node micromodulus factor or NULL */
    double damping;
    /* state, caller-owned */
    double* U;
    double* V;
    double* vbuf;
    double* ug;                /* [n][npt][3] */
    double* eed;               /* [n] elastic energy density */
    double ke, ee;             /* energies of the last RK4 step */
} or_model;

/* pdDataManager3.cpp:1706-1799 (SetGaussianPointsValue): 1-D abscissae and
 * weights of the n-point rule; returns the count written (n, or 1). */
int or_gauss_1d(int n, double* absc, double* wts);

/* pdDataManager2.cpp:72-104: Gauss point coordinates [n][n1^3][3] and the
 * per-point axis weights [n1^3][3]. */
void or_gauss_points(int64_t n, const double* x, double dx, int n1, double* xg, double* gw);

/* pdDataManager2.cpp:12-70 + pdDataManager3.cpp:637-685,1573-1704: family
 * CSR (ascending ids).  With col == NULL only row_ptr is filled.  min_bond
 * receives _minBondLength.  Returns total halves, or -1 if cap is too small. */
int64_t or_bond_search(int64_t n, const double* x, double dx, double delta,
                       int64_t* row_ptr, int32_t* col, int64_t cap, double* min_bond);

/* Project rule for pdSlit: mark family entries whose segment crosses any of
 * the rectangles slits[k] = {x1lo,x1hi,x2lo,x2hi,x3lo,x3hi}. */
void or_slit_mark(int64_t n, const double* x, const int64_t* row_ptr, const int32_t* col,
                  int nslit, const double* slits, uint8_t* broken);

/* pdDataManager2.cpp:118-171: contributor CSR; cb_idx NULL = count only. */
int64_t or_mls_contributors(int64_t n, const double* x, const int64_t* row_ptr, const int32_t* col,
                            double rw, int64_t* cb_ptr, int32_t* cb_idx);

/* pdDataManager2.cpp:173-256 with GetBasis/GetWeight (:1547-1578) and
 * pdMatrix::Gauss (pdMatrix.cpp:251-391).  Returns 0, or -(node+1) for a
 * singular moment matrix. */
int64_t or_mls_coeff(int64_t n, const double* x, const double* xg, int npt, const int64_t* cb_ptr,
                     const int32_t* cb_idx, double rw, double* coeff);

/* pdDataManager.cpp:1340-1473, pdDataManager2.cpp:1353-1485.  Writes bE[n]
 * and returns the full-sphere family count. */
int or_bdry_eff(const or_model* m, const int* dims, const double* center, double* bE);

/* pdDataManager.cpp:2402-2495 (with UpdateIntgPointStatusWithBC :2604-2703). */
void or_gather(or_model* m, double t, const double* us);

/* pdDataManager.cpp:1767-1992 + UpdateNodeStatusWithBC :2497-2602, plus the
 * project's traction load.  k[3n] out. */
void or_force_stage(or_model* m, double dts, double t, const double* us, double* k);

/* pdDataManager2.cpp:410-439 + pdDataManager.cpp:1994-2134. */
void or_rk4_step(or_model* m, double dt, double t);

/* Adaptive-trapezoid (AI) force stage: the ai_on branch of
 * CalcBondBasedMotionRK4 (pdDataManager.cpp:1886-1915) with
 * CalcBondForceIntg (pdDataManager2.cpp:1227-1291) and the nested trapezoid
 * rule of pdIntgManager (pdIntgManager.cpp:49-451; integrand
 * pdIntgManager2.cpp:92-310), node by node in the reference's order.  The
 * regions of every family entry come from reg_ptr / regs (the layout of
 * pd_ai_plan: 24 bytes per region, a, b, axis[3], lim[4], flags); with
 * m->mls the displacement of a region's k-th point is the MLS sum over node
 * j's contributors with coefficient list entry k (tab_ptr [n+1] entries,
 * tab_coeff [entry][contributor]); a boundary-condition node j gives its
 * prescribed value in flagged DISPL / DISPLGRAD directions.  Without MLS
 * every family node carries a displacement gradient G and eta = G xi.  A
 * point past the critical stretch gives no force, breaks the bond for both
 * nodes (ai_broken [entries], updated in place) and adds 1 to dmg [n].
 * k [3n] out, as or_force_stage. */
void or_ai_force_stage(or_model* m, int trap, const int64_t* reg_ptr, const void* regs, const int64_t* tab_ptr,
                       const double* tab_coeff, uint8_t* ai_broken, int32_t* dmg, double dts, double t,
                       const double* us, double* k);

/* pdSolve.cpp:195-527 restated as an operator on the 3n system: free rows
 * sum c*V_j*xi xi^T/r^3 (x_i - x_j) over unbroken family members, with
 * prescribed columns masked; prescribed rows are identity. */
void or_static_apply(const or_model* m, double t, const double* x, double* y);
/* right-hand side: prescribed values, the moved prescribed columns and the
 * traction body-force density (project rule). */
void or_static_rhs(const or_model* m, double t, double* b);

/* plain FP64 CG on the static system; returns iterations or -1. */
int or_static_cg(const or_model* m, double t, const double* b, double* x, double rtol, int maxit, double* relres);

/* Project rule (no counterpart in the reference): runs nsteps of
 * or_rk4_step from the model's state at t0 (t += dt before each step),
 * keeping every stage's inputs, then accumulates in reverse the gradient
 * gradf [n] of J with respect to spring_factor, for lamU/lamV [n][3] = dJ/dU,
 * dJ/dV of the final state (lamV may be NULL).  The model is left at the
 * final state.  Returns 0, or -1 when memory runs out. */
int or_adjoint_grad(or_model* m, double dt, double t0, int nsteps, const double* lamU, const double* lamV,
                    double* gradf);

#ifdef __cplusplus
}
#endif
#endif
