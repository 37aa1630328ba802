/*
 * pdmtel_b200.h — C ABI of the B200 pdMTEL hot path (libpdmtel_b200.so).
 *
 * Plain pointers and sizes only.  Every entry point returns an int status:
 * PD_OK (0) or a negative PD_ERR_* code; pd_last_error() gives a message.
 * Host arrays are caller-owned and copied; device memory is owned by the
 * context.  One CUDA stream per context (given in pd_problem.stream, or
 * created).  A context is not thread-safe; distinct contexts may be used from
 * distinct threads.
 *
 * Vectors of node quantities use the reference's row order (3*i + a, the
 * "_rowOfNode" layout of pdDataManager.cpp:1089-1091).  Gauss-point
 * displacements are [node][point][3] (the pdNode Gaussian point list order,
 * pdDataManager2.cpp:72-104).
 */
#ifndef PDMTEL_B200_H
#define PDMTEL_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PD_ABI_VERSION 1

enum pd_status {
    PD_OK = 0,
    PD_ERR_ARG = -1,       /* bad argument or call order */
    PD_ERR_OOM = -2,       /* device or host allocation failed */
    PD_ERR_CUDA = -3,      /* CUDA runtime error */
    PD_ERR_TIMEOUT = -4,   /* a bounded device wait gave up */
    PD_ERR_SINGULAR = -5,  /* singular MLS moment matrix (pdMatrix.cpp:297,335) */
    PD_ERR_CAPACITY = -6,  /* caller buffer too small */
    PD_ERR_NOCONV = -7,    /* iterative solve did not reach the tolerance */
    PD_ERR_NODEV = -8      /* no CUDA device */
};

/* boundary-condition types, pdDataManager.h:231 / pdBdryCondition.h:25 */
enum pd_bc_type { PD_BC_DISPL = 1, PD_BC_VELOC = 2, PD_BC_DISPLGRAD = 3, PD_BC_TRACTION = 4 };
/* volume integration scheme, pdDataManager.cpp:571-730 */
enum pd_integration {
    PD_INTG_CCI = 0,
    PD_INTG_FGI = 1,
    /* adaptive trapezoid over the family cell cut by the horizon sphere
     * (ai_on, pdIntgManager types 1-3); intg_point is the trapezoid index
     * (1..3: 2, 3 or 5 points per direction); data from pd_set_ai */
    PD_INTG_AI = 2
};
/* arithmetic of the force / gather / matvec kernels */
enum pd_precision {
    PD_PREC_FP64 = 0,  /* the drop-in: bit-faithful to the reference CPU path */
    PD_PREC_FP32C = 1, /* FP32 forces, compensated sums, FP64 state */
    PD_PREC_FP64A = 2  /* FP64 with the bond extension p - r formed as
                          (2 xi.eta + eta.eta) / (p + r): the same function
                          without the cancellation of p - r at small strain
                          (rounding ~eps instead of ~eps/strain); not
                          bit-faithful to the reference */
};

/* bond-based (PMB) material, pdMaterialBond.cpp:8-11; spring = 18K/(pi d^4)
 * as pdDataManager.cpp:1314 computes it */
typedef struct pd_material {
    double spring;
    double density;
    double ecrit;
    double grav[3];
} pd_material;

/* pdBdryCondition (pdBdryCondition.h:25-67): value[3] for DISPL, VELOC and
 * TRACTION, value[9] (row-major gradient) for DISPLGRAD; load_type 1 = ramp */
typedef struct pd_bc {
    int32_t type;
    int32_t dir[3];
    double value[9];
    double end_time;
    double load_type;
} pd_bc;

typedef struct pd_problem {
    int64_t num_nodes;
    const double* coords;        /* [N][3] (pdDataManager.cpp:846-907) */
    const int32_t* mat_id;       /* [N] material index (0-based) */
    const int32_t* bc_id;        /* [N] bc index or -1; NULL = none */
    int32_t num_materials;
    const pd_material* materials;
    int32_t num_bcs;
    const pd_bc* bcs;
    double grid_spacing;         /* _gridSpacing */
    double horizon;              /* _horizon */
    int32_t integration;         /* pd_integration */
    int32_t cci_modified;        /* _cciMdf */
    int32_t intg_point;          /* 1-D Gauss order n (FGI); n^3 points */
    const double* abscissae;     /* [n], pdDataManager3.cpp:1706-1799 */
    const double* weights;       /* [n] */
    double damping;              /* _dampCoeff */
    int32_t num_slits;           /* slit rectangles x1lo x1hi x2lo x2hi x3lo x3hi */
    const double* slits;
    const double* spring_factor; /* [N] per-node micromodulus factor, or NULL */
    void* stream;                /* cudaStream_t to run on, or NULL */
} pd_problem;

typedef struct pd_ctx pd_ctx;

int pd_abi_version(void);
const char* pd_last_error(void);
/* number of CUDA devices visible (0 on a machine without a GPU) */
int pd_device_count(int* count);

/* Allocates the device arrays of one problem (pdDataManager state of
 * pdDataManager.h:169-234).  Replaces the data set up by InitNode and
 * InitMaterial (pdDataManager.cpp:813-1098,1297-1338). */
int pd_ctx_create(const pd_problem* problem, pd_ctx** out);
int pd_ctx_destroy(pd_ctx* ctx);
/* the CUDA stream of the context (cudaStream_t) */
int pd_ctx_stream(pd_ctx* ctx, void** stream);
int pd_sync(pd_ctx* ctx);

/* Cell-binned, Morton-ordered family search on the device.  Replaces
 * pdDataManager::InitBond (pdDataManager2.cpp:12-70) with its cube-distance
 * test (pdDataManager3.cpp:637-685,1573-1704); the family list of every
 * node is in ascending id order, as the reference's is.  Slit rectangles
 * mark crossing bonds broken.  Outputs the number of family entries
 * (2 x bonds) and _minBondLength. */
int pd_bond_search(pd_ctx* ctx, int64_t* num_halves, int64_t* num_broken, double* min_bond_length);
/* Copies the family CSR out (row_ptr [N+1], col [H], broken [H] or NULL). */
int pd_get_family(pd_ctx* ctx, int64_t* row_ptr, int32_t* col, uint8_t* broken);
/* Installs a family CSR built elsewhere (same layout); broken may be NULL. */
int pd_set_family(pd_ctx* ctx, const int64_t* row_ptr, const int32_t* col, const uint8_t* broken);

/* Boundary-effect factors (pdNode::SetBdryEffFactor, from
 * pdDataManager::InitBdryEffectFactor pdDataManager.cpp:1340-1473). */
int pd_set_bdry_eff(pd_ctx* ctx, const double* bdry_eff);
/* MLS contributors and coefficients from InitIntegrationPoint
 * (pdDataManager2.cpp:118-256): cb_ptr [N+1], cb_idx, coeff laid out per
 * node as [point][contributor]. */
int pd_set_mls(pd_ctx* ctx, const int64_t* cb_ptr, const int32_t* cb_idx, const double* coeff);
/* The same MLS data computed on the device from the context's family (the
 * contributor rule of pdDataManager2.cpp:118-171: the node, then family
 * members within rw, within 1.5 rw when fewer than 10) and coordinates, or
 * from mls_coords ([N][3] host, may be NULL: each node's coordinates in the
 * frame its MLS is solved in, e.g. a batch specimen's own frame).  Moment
 * matrices and their full-pivot solve follow pdDataManager2.cpp:173-256 and
 * pdMatrix.cpp:251-391 operation for operation; only the spline weight's
 * d^3 and d^4 (glibc pow in the reference, off the correctly rounded value
 * for ~4e-4 of the arguments) are rounded once, so the coefficients equal
 * the reference's where those agree and differ by the moment matrix's
 * round-off elsewhere.  PD_ERR_SINGULAR on a singular moment matrix.
 * *num_contrib (may be NULL) receives the number of contributor entries. */
int pd_mls_setup(pd_ctx* ctx, double rw, const double* mls_coords, int64_t* num_contrib);
/* The context's MLS data out in the layout of pd_set_mls: cb_ptr [N+1],
 * cb_idx [entries] and coeff [entries x points] (either may be NULL). */
int pd_get_mls(pd_ctx* ctx, int64_t* cb_ptr, int32_t* cb_idx, double* coeff);
/* Adaptive-trapezoid (AI) integration (pdDataManager::CalcBondForceIntg,
 * pdDataManager2.cpp:1227-1291; pdIntgManager.cpp:49-3491).  A bond's force is
 * a sum of regions, each a nested trapezoid rule: the outer direction axis[0]
 * over [a, b], the middle direction axis[1] between the limit functions
 * lim[0], lim[1] of the outer value, the inner direction axis[2] between
 * lim[2], lim[3] of the outer and middle values.  Limit codes (dx spacing,
 * x_j the family node relative to node i, delta the horizon):
 *   middle: 2 axis + side          x_j[axis] -/+ dx/2 (side 0 low, 1 high)
 *           8 + 4 (3 A + B) + 2 side + sign
 *                                  +/- sqrt(r^2 - t^2) (0 where negative),
 *                                  r^2 = delta^2 - (x_j[C] -/+ dx/2)^2, t the
 *                                  outer value, C the axis other than A, B
 *   inner:  2 axis + side          x_j[axis] -/+ dx/2
 *           8 + 2 axis + sign      +/- sqrt(delta^2 - t^2 - s^2) (0 where
 *                                  negative), s the middle value
 * sign 1 is +.  PD_AI_ASSIGN on a bond's first region: the force is that
 * region's integral (the reference writes it), else the regions are added to
 * a sum that starts at 0.0. */
#define PD_AI_ASSIGN 1
typedef struct pd_ai_region {
    double a, b;
    uint8_t axis[3];
    uint8_t lim[4];
    uint8_t flags;
} pd_ai_region;
/* The regions of every full-family entry (pd_get_family order; the bond
 * classification of CalcBondForceIntg and the case analysis of
 * pdIntgManager::AdaptiveIntegration, pdIntgManager.cpp:523-3482, from the
 * coordinates coords [N][3]): reg_ptr [entries + 1], regions (NULL to size
 * the list: *num_regions receives the count; PD_ERR_CAPACITY when capacity is
 * smaller).  Host only; needs no device. */
int pd_ai_plan(int64_t num_nodes, const double* coords, const int64_t* row_ptr, const int32_t* col,
               double grid_spacing, double horizon, int64_t* reg_ptr, pd_ai_region* regions, int64_t capacity,
               int64_t* num_regions);
/* The per-node MLS coefficient lists of the AI form (InitIntegrationPoint's
 * trapezoid pass, pdDataManager2.cpp:257-300, and
 * pdIntgManager::InitMLSCoeff, pdIntgManager2.cpp:1879-1939): node j's list
 * holds the coefficients of the trapezoid points of the bonds i -> j in the
 * order the reference's setup pass visits them, and the force pass reads
 * entry k for a region's k-th point, whichever bond it integrates.  Only the
 * entries the force pass can reach are kept: tab_ptr [N+1] (entries per node,
 * cumulative), tab_coeff [entry][contributor of the node] (NULL to size:
 * *num_coeff receives the count of doubles).  cb_ptr / cb_idx: the MLS
 * contributors (pd_get_mls layout); rw the support radius; trap_index 1..3.
 * PD_ERR_SINGULAR with the node in *bad_node on a singular moment matrix.
 * Host only. */
int pd_ai_mls_table(int64_t num_nodes, const double* coords, const int64_t* row_ptr, const int32_t* col,
                    const int64_t* reg_ptr, const pd_ai_region* regions, double grid_spacing, double horizon,
                    int trap_index, const int64_t* cb_ptr, const int32_t* cb_idx, double rw, int64_t* tab_ptr,
                    double* tab_coeff, int64_t capacity, int64_t* num_coeff, int64_t* bad_node);
/* Upload the AI data to a context created with PD_INTG_AI, after its family:
 * the regions of every full-family entry (pd_ai_plan layout) and, with
 * mls = 1, the MLS contributors cb_ptr / cb_idx (pd_get_mls layout) and
 * tables (pd_ai_mls_table layout).  A new family drops the AI data.  With
 * mls = 0 every family node carries a displacement-gradient boundary
 * condition and eta = G xi (pdIntgManager2.cpp:211-235).  With MLS, a family
 * node with a boundary condition gives its prescribed value in the DISPL /
 * DISPLGRAD directions it flags; its other directions take the MLS value
 * (the reference reads an unset local there).
 * A bond whose point passes the critical stretch is broken from then on for
 * both of its nodes (pdIntgManager2.cpp:301-308); the FP64 arithmetic only. */
int pd_set_ai(pd_ctx* ctx, int mls, const int64_t* reg_ptr, const pd_ai_region* regions, const int64_t* cb_ptr,
              const int32_t* cb_idx, const int64_t* tab_ptr, const double* tab_coeff);
/* The AI form's damage state: broken [full-family entries] (the family's
 * flags plus the bonds the AI integrand broke) and count [N], the points of
 * node i past the critical stretch in the last step (pdNode's damaged-bond
 * count, pdIntgManager2.cpp:308; reset by pdDataManager::InitDynamicSolve,
 * pdDataManager2.cpp:426).  Either may be NULL; other schemes report their
 * family's flags and zero counts. */
int pd_get_damage(pd_ctx* ctx, uint8_t* broken, int32_t* count);
/* number of MLS contributor entries held (0 without MLS data) */
int pd_mls_size(pd_ctx* ctx, int64_t* num_contrib);

/* The areal-force-density sums of pdSolve::PostAFD (pdSolve.cpp:810-834,
 * pdDataManager3.cpp:442-635,1101-1223, replacing CalcForceOfPlusSpace).
 * U [N][3] and bdry_eff [N] (host) are the nodal displacements and
 * boundary factors PostAFD reads from a Tecplot dump; the Gauss-point
 * displacements are derived from U as PostAFD derives them
 * (CalcApproxDispl, pdDataManager.cpp:2704-2752: flagged directions of
 * boundary-condition nodes stay zero).  Item k (node item_i, source
 * item_s, direction item_dir 1..3) receives in force[3k..3k+2] the sum, over
 * the family members j of node item_i (ascending id) with x_j >= x_source
 * along the direction, of the bond force integrated over cell j: the fixed
 * Gauss rule nested as pdIntgManager::CalcConfigurationType3 nests it, or
 * the one-point CCI force with the node volume.  The caller adds the items
 * of a source into its stress tensor (x ds, in the reference's order). */
int pd_afd(pd_ctx* ctx, const double* U, const double* bdry_eff, int64_t num_items, const int64_t* item_i,
           const int64_t* item_s, const int32_t* item_dir, double* force);

/* Arithmetic of the subsequent force/gather/step calls (pd_precision). */
int pd_set_precision(pd_ctx* ctx, int precision);
/* Whether the elastic-energy diagnostic (pdDataManager2.cpp:1340-1342,
 * pdDataManager.cpp:2096-2115) is accumulated; on by default. */
int pd_set_energy(pd_ctx* ctx, int on);

/* Nodal state U and V ([3N] each; either may be NULL).  Setting the state
 * also sets the velocity buffer to V (InitDynamicSolve).  Like the
 * reference's pdNode::SetU1..3, it leaves the Gauss-point displacements
 * alone: the next step's first stage reads the ones the last gather derived.
 * Call pd_gather(ctx, t, NULL) to derive them from the new U. */
int pd_set_state(pd_ctx* ctx, const double* U, const double* V);
int pd_get_state(pd_ctx* ctx, double* U, double* V);
int pd_get_vbuf(pd_ctx* ctx, double* vbuf);
int pd_set_gauss_displ(pd_ctx* ctx, const double* ug);
int pd_get_gauss_displ(pd_ctx* ctx, double* ug);
/* per-node elastic energy density of the current step */
int pd_get_energy_density(pd_ctx* ctx, double* eed);

/* pdDataManager::InitDynamicSolve (pdDataManager2.cpp:410-439). */
int pd_init_dynamic(pd_ctx* ctx);
/* pdDataManager::CalcIntgPointDisplRK4 (pdDataManager.cpp:2402-2495): the
 * Gauss-point displacements from trial nodal displacements us [3N] (host);
 * us == NULL uses the nodal state U. */
int pd_gather(pd_ctx* ctx, double time, const double* us);
/* pdDataManager::CalcBondBasedMotionRK4 (pdDataManager.cpp:1767-1992): adds
 * the bond forces of trial displacements us [3N] to the velocity buffer,
 * applies the boundary conditions (UpdateNodeStatusWithBC :2497-2602) and
 * writes k = vbuf*dt into k_out [3N] (may be NULL). */
int pd_force_stage(pd_ctx* ctx, double dt, double time, const double* us, double* k_out);
/* pdDataManager::RK4 (pdDataManager.cpp:1994-2134), preceded by
 * InitDynamicSolve; ke/ee (may be NULL) receive the kinetic and elastic
 * energies of the step (pdSolve.cpp:85-91). */
int pd_rk4_step(pd_ctx* ctx, double dt, double time, double* ke, double* ee);
/* nsteps consecutive RK4 steps on the device, the time advancing as
 * pdSolve.cpp:59-61 advances it (t += dt before each step, from t0).  The
 * steps are captured once into a CUDA graph and replayed. */
int pd_rk4_steps(pd_ctx* ctx, double dt, double t0, int nsteps);
/* The same through host buffers: U,V in [3N] are uploaded, nsteps run and
 * the new state written to U_out,V_out.  When U_in differs from the device's
 * displacement, the Gauss-point displacements are first derived from U_in at
 * t0 (pd_gather), so the steps continue from U_in exactly as from a state the
 * device reached by stepping; when it is the same (a round trip of the
 * previous call's output), nothing is recomputed. */
int pd_rk4_steps_host(pd_ctx* ctx, double dt, double t0, int nsteps, const double* U_in, const double* V_in,
                      double* U_out, double* V_out);
/* number of Gauss-point force evaluations of one RK4 stage (unbroken
 * family entries x points per node, CCI: one per entry) */
int pd_evals_per_stage(pd_ctx* ctx, int64_t* evals);
/* Back to the state InitNode and SetGaussianPoint leave (pdDataManager.cpp:
 * 1062-1087, pdDataManager2.cpp:93-96): displacements, velocities, the
 * velocity buffer and every Gauss-point displacement zero. */
int pd_reset_state(pd_ctx* ctx);
/* One RK4 step like pd_rk4_step, with CUDA events on the context's stream
 * around every kernel; ms[0..3] receive the summed device time of the force,
 * gather, stage-epilogue and remaining kernels of the step. */
int pd_profile_step(pd_ctx* ctx, double dt, double time, double* ms);

/* ---- Bond search for callers that cannot allocate device memory ----
 *
 * No counterpart in the reference.  pd_bond_search needs a context, and a
 * context calls cudaMalloc.  Some hosts cannot: an application that hands
 * all device memory to its own pool at start-up and forbids allocations
 * afterwards, or a plugin whose memory is owned by the host program, or a
 * loop that must not block on cudaMalloc's implicit synchronisation.  This
 * entry point performs the same search (same membership test, same
 * ascending-id family order, same slit marks) into buffers the caller
 * provides, and allocates nothing: its working memory is one fixed array of
 * PD_NOALLOC_SCRATCH_BYTES in device memory, part of the library image, which
 * every GPU that loads the library holds until the process exits.
 *
 * Limits: at most PD_NOALLOC_MAX_NODES nodes, PD_NOALLOC_MAX_CELLS search
 * cells (bounding box / (horizon + spacing), rounded up, per axis, multiplied)
 * and PD_NOALLOC_MAX_SLITS slits; larger problems return PD_ERR_CAPACITY.
 *
 * coords: device, [n][3].  row_ptr: device, [n+1], always written.  col and
 * broken (broken may be NULL): device, [capacity]; when the family is larger
 * than capacity the call returns PD_ERR_CAPACITY after writing row_ptr and
 * *num_halves, so the caller can size col and call again.  slits: host,
 * [num_slits][6].  stream: a cudaStream_t or NULL.  The call waits for its
 * stream several times (it reads the bounding box, the family size and the
 * longest family back to the host between its launches) and returns with the
 * stream idle.  A non-finite coordinate returns PD_ERR_ARG; the cell count is
 * checked axis by axis, so a horizon tiny next to the extent returns
 * PD_ERR_CAPACITY instead of overflowing.
 *
 * The first call on each device looks up the array's device address
 * (cudaGetSymbolAddress) with that device current; make that first call
 * before any stream capture.  All calls share the one array and it keeps the
 * last call's contents (the call clears what must start at zero): calls that
 * overlap on the GPU, from several threads or streams, race and must be
 * serialised by the caller. */
#define PD_NOALLOC_MAX_NODES 65536
#define PD_NOALLOC_MAX_CELLS 65536
#define PD_NOALLOC_MAX_SLITS 16
#define PD_NOALLOC_SCRATCH_BYTES 2622360
int pd_bond_search_noalloc(const double* coords, int64_t num_nodes, double grid_spacing, double horizon,
                           int32_t num_slits, const double* slits, int64_t* row_ptr, int32_t* col, uint8_t* broken,
                           int64_t capacity, void* stream, int64_t* num_halves, double* min_bond_length);

/* Prepares the static operator (done by the first static call otherwise):
 * decides whether it runs as a lattice stencil (PD_OPT_STATIC_STENCIL) and
 * builds the stencil; *stencil (may be NULL) receives 1 if it does. */
int pd_static_prepare(pd_ctx* ctx, int* stencil);
/* Linearised stiffness operator of pdSolve::AssembleEquation (pdSolve.cpp:
 * 195-527) applied matrix-free: free rows sum c V_j xi xi^T / r^3 (x_i - x_j)
 * over the unbroken family with prescribed columns masked, prescribed rows
 * return x.  time selects VELOC values (val*time, pdSolve.cpp:245-262). */
int pd_static_matvec(pd_ctx* ctx, double time, const double* x, double* y);
/* right-hand side: prescribed values, moved prescribed columns and the
 * traction load (value*factor/grid_spacing on TRACTION nodes). */
int pd_static_rhs(pd_ctx* ctx, double time, double* b);
/* Matrix-free CG on the static system (the dense Gauss-Jordan of
 * pdSolve::Gauss pdSolve.cpp:545-673 is replaced).  PD_PREC_FP64: FP64 CG;
 * PD_PREC_FP32C: the iterations' matvec in FP32 (FP64 vectors, dot products
 * and node sums), refined in FP64 by replacing the residual with the true
 * b - K x whenever it has fallen 100-fold and at convergence ("reliable
 * updates"); convergence is judged on the FP64 true residual.  x [3N] is the
 * initial guess in and the solution out.  iters/relres may be NULL. */
int pd_static_solve(pd_ctx* ctx, double time, int precision, double rtol, int maxit, double* x, int* iters,
                    double* relres);

/* ---- Tuning options (no counterpart in the reference) ----
 * None of them changes a result (PD_OPT_STATIC_PRECOND: beyond the solve's
 * tolerance); they change launch shapes only.
 * PD_OPT_F64_LANES_BELOW: the FP64 Gauss-point force runs eight lanes per
 *   node (same arithmetic, same order) when the problem has fewer nodes than
 *   this, one thread per node otherwise.  Default 131072.
 * PD_OPT_TILE: the node work order walks lattice tiles of 2^bx x 2^by x 2^bz
 *   nodes, value = bx | by << 8 | bz << 16 (1 <= bx <= 6, by, bz <= 6).
 *   Default 8 x 4 x 4.
 * PD_OPT_PERSIST_BLOCKS_PER_SM: blocks per SM of the persistent launch (0:
 *   as many as fit).
 * PD_OPT_PERSIST_FORCE_CHUNK / _GATHER_CHUNK: work items a block takes from
 *   the queue at a time (multiples of 128; defaults 128 and 256).
 * PD_OPT_STATIC_STENCIL: 1 (default) lets the static operator run as a
 *   lattice stencil when the problem is a complete box with one material,
 *   no broken bond and stencil-shaped families (checked); 0 keeps the
 *   family-list kernel.
 * PD_OPT_GATHER_PER_POINT: 1 runs the FP32-form MLS gather with one thread
 *   per (node, Gauss point), 0 (default) with one per four points.
 * PD_OPT_FORCE_TILE: the FP32-form force (2x2x2 points, nodes on one
 *   lattice) stages lattice tiles of tx x ty x tz positions and their halo
 *   in shared memory, value = tx | ty << 8 | tz << 16 (tx even, 32 to 256
 *   pairs of positions per tile); 0 (default) reads neighbours from global
 *   memory.  Reset to 0 whenever the family changes.
 * PD_OPT_FORCE_QUAD: 1 runs the FP32-form force with four nodes per thread
 *   (nodes on one lattice, one material, no critical stretch within reach;
 *   otherwise ignored); 0 (default) with two.
 * PD_OPT_GATHER_SELL: 1 keeps a sliced-ELLPACK copy of the FP32 gather's
 *   contributor lists and coefficients (16 nodes of the work order side by
 *   side per contributor slot: coalesced loads; 2x2x2 points), 0 (default)
 *   reads the CSR lists.  Costs a second FP32 copy of the coefficients.
 * PD_OPT_PERSIST_WAIT_US: how long a grid barrier of the persistent launch
 *   waits before it gives up (default 4 s; 1 ms to 60 s).
 * PD_OPT_PERSIST_TEST_STALL: 1 makes block 0 of the persistent launch skip
 *   its first barrier, so that every wait there runs out and the call
 *   returns PD_ERR_TIMEOUT; for tests of that path.  0 by default.
 * PD_OPT_FORCE_STENCIL: 1..4 runs the FP32-form force on the lattice
 *   stencil: the family of every node becomes a bit mask over one list of
 *   lattice offsets, the gather stores the node blocks chunk-major, and a
 *   block covers 16 x-adjacent node pairs by (8x1, 4x2, 2x4, 1x8) rows x
 *   layers for the values 1..4.  Needs 2x2x2 points, one material and a
 *   complete box lattice whose node ids are x + nx (y + ny z) (checked on
 *   the device: PD_ERR_ARG otherwise).  Takes precedence over the other
 *   force variants; 0 (default) turns it off.  Reset to 0 whenever the
 *   family changes.  Same results bit for bit as the other FP32 kernels
 *   when no critical stretch is within reach (with one, those form bond
 *   vectors from FP32 hi/lo coordinate splits instead of lattice offsets,
 *   and the results agree to FP32 rounding).
 *   Turning it on or off changes the layout of the node blocks that
 *   pd_gather stores for pd_force_stage: gather again after the change.
 *   Each force stage is two launches on the context's stream: a pass that
 *   evaluates every Gauss point with the strain series alone, then a pass
 *   that redoes, with the exact form where needed, only the tiles in which
 *   a point left the series range (one byte per tile, kept by the context).
 * PD_OPT_GATHER_STENCIL: 1 lets the FP32-form gather (one thread per four
 *   points) take every node's MLS contributors from a pattern of id offsets
 *   (nodes whose lists are translates of each other share one; kept with
 *   the context and rebuilt by pd_set_mls) instead of its list, so the
 *   contributor loads no longer wait on an index load from memory.  Same
 *   contributors in the same order: same results bit for bit.  Refused
 *   (PD_ERR_ARG) when the distinct patterns would hold more than a quarter
 *   of all list entries (at least 4M allowed, at most 64M); 0 (default)
 *   reads the lists.
 * PD_OPT_STATIC_PRECOND: 1 (default) preconditions the static CG with the
 *   inverses of the operator's 3x3 diagonal blocks (block Jacobi); 0 runs
 *   plain CG.  Changes the iterates, not the solution beyond the tolerance.
 * PD_OPT_STATIC_SPLIT: the FP64 lattice-stencil operator in the split form
 *   K x = D_i x_i - sum_o W_o x_(i+o) (three FMAs per bond instead of ten;
 *   the same operator to FP64 rounding) with 2, 4 (default) or 8 nodes per
 *   thread along z; 0 runs the difference form.  No effect on the FP32
 *   operator, on spring factors (pd_set_spring_factor) or off the stencil.
 * PD_OPT_STATIC_F32_BELOW: v; the FP32C static solve iterates with the FP64
 *   operator until the relative residual is below 1/v, then with the FP32
 *   one (default 10: below 0.1); 0 uses the FP32 operator from the start.
 * PD_OPT_ADJOINT_VJP32: 1 makes the reverse sweep of an FP32C forward run
 *   (pd_adjoint_backward) evaluate its point terms in FP32 (faster; the
 *   family sums of a smooth adjoint cancel, so its gradient is good to about
 *   1e-3); 0 (default) keeps them FP64 on the FP32C tape. */
enum {
    PD_OPT_F64_LANES_BELOW = 1,
    PD_OPT_TILE = 2,
    PD_OPT_PERSIST_BLOCKS_PER_SM = 3,
    PD_OPT_PERSIST_FORCE_CHUNK = 4,
    PD_OPT_PERSIST_GATHER_CHUNK = 5,
    PD_OPT_STATIC_STENCIL = 6,
    PD_OPT_GATHER_PER_POINT = 7,
    PD_OPT_FORCE_TILE = 8,
    PD_OPT_FORCE_QUAD = 9,
    PD_OPT_PERSIST_WAIT_US = 10,
    PD_OPT_PERSIST_TEST_STALL = 11,
    PD_OPT_GATHER_SELL = 12,
    PD_OPT_FORCE_STENCIL = 13,
    PD_OPT_GATHER_STENCIL = 14,
    PD_OPT_STATIC_PRECOND = 15,
    PD_OPT_STATIC_SPLIT = 16,
    PD_OPT_STATIC_F32_BELOW = 17,
    PD_OPT_ADJOINT_VJP32 = 18
};
int pd_set_option(pd_ctx* ctx, int option, int64_t value);
int pd_get_option(pd_ctx* ctx, int option, int64_t* value);

/* ---- Batching: persistent stepping and the autotuner (no counterpart in the
 * reference) ----
 * A batch of specimens is one context whose family has no bond between
 * specimens (the host layer places them apart), so every entry point above
 * steps all specimens at once.  pd_rk4_steps_persistent runs nsteps steps of
 * the FP32-compensated form in ONE cooperative launch (every block resident;
 * work taken from per-phase queues; grid barriers between the force and the
 * gather phases give up after 4 s with PD_ERR_TIMEOUT), captured into a CUDA
 * graph per (dt, nsteps, launch shape).  Needs PD_PREC_FP32C, 2x2x2 Gauss
 * points and energy accumulation off; same result bit for bit as
 * pd_rk4_steps.  Synchronous. */
/* Declares that the node ranges offsets[b] .. offsets[b + 1] - 1 (b < nbox,
 * offsets[0] = 0, offsets[nbox] = the node count) each form a complete box
 * lattice whose node ids follow x + nx (y + ny z) from the range's first
 * node, as the specimens of a batch do; the box dimensions are read from the
 * coordinates.  PD_OPT_FORCE_STENCIL then runs the lattice-stencil FP32 force
 * on every box.  nbox = 0 returns to one box.  PD_ERR_ARG when a range is
 * not such a box. */
int pd_set_boxes(pd_ctx* ctx, int nbox, const int64_t* offsets);
int pd_rk4_steps_persistent(pd_ctx* ctx, double dt, double t0, int nsteps);
typedef struct pd_tune_result {
    int64_t tile;          /* PD_OPT_TILE value kept */
    int32_t persistent;    /* 1: the persistent launch was fastest */
    int32_t blocks_per_sm; /* PD_OPT_PERSIST_BLOCKS_PER_SM kept */
    int32_t force_chunk, gather_chunk;
    int32_t trials;
    double ms_per_step;    /* device time per step of the kept shape */
    int32_t gather_per_point; /* PD_OPT_GATHER_PER_POINT kept */
    int32_t pad;
    int64_t force_tile;       /* PD_OPT_FORCE_TILE kept */
    int32_t force_quad;       /* PD_OPT_FORCE_QUAD kept */
    int32_t gather_sell;      /* PD_OPT_GATHER_SELL kept */
    int32_t force_stencil;    /* PD_OPT_FORCE_STENCIL kept */
    int32_t gather_stencil;   /* PD_OPT_GATHER_STENCIL kept */
} pd_tune_result;
/* Times candidate launch shapes (node-order tiles, the FP32 gather variants:
 * per point, SELL copy, contributor patterns;
 * the FP32 force variants: lattice stencil, four nodes per thread,
 * shared-memory force tiles;
 * for the persistent launch blocks per SM and queue chunks) over `steps`
 * steps each from the current state, keeps the fastest in the context and
 * restores the state. */
int pd_autotune(pd_ctx* ctx, double dt, int steps, pd_tune_result* out);

/* ---- Differentiation: gradient with respect to a per-node micromodulus ----
 *
 * No counterpart in the reference (its spring constant is per material with
 * the min(c_i, c_j) pair rule, pdDataManager.cpp:1926).  With spring factors
 * f the pair constant is min(c_i, c_j) * (f_i + f_j) / 2, which is
 * differentiable in f; f = exp(m) gives a log-micromodulus field m. */
/* replace the per-node spring factors f [N] (host, positive) */
int pd_set_spring_factor(pd_ctx* ctx, const double* f);
/* Forward half of the adjoint pair: nsteps RK4 steps of the scheme of
 * pdDataManager::RK4 (pdDataManager.cpp:1994-2134) from the current state at
 * time t0, storing (U, V, Gauss-point displacements, time) every
 * checkpoint_every steps in the context.  The state ends at step nsteps.
 * The steps run in the context's precision: FP64 (PD_PREC_FP64A stays
 * FP64A), or at PD_PREC_FP32C the
 * compensated FP32 step (checkpoints then hold its node blocks, so the
 * reverse sweep recomputes the forward bit for bit).
 * FGI (Gauss-point) scheme only. */
int pd_adjoint_forward(pd_ctx* ctx, double dt, double t0, int nsteps, int checkpoint_every);
/* Backward half: the vector-Jacobian product of the last forward run.
 * lam_U, lam_V [3N] (host; lam_V may be NULL) are dJ/dU and dJ/dV of the
 * final state; grad_f [N] (host) receives dJ/df.  Each checkpointed segment
 * is recomputed with its stage inputs kept, then reversed stage by stage
 * (force VJP as two gathers, transposed MLS gather); deterministic, no
 * atomics.  The state is left at the start of the forward run. */
int pd_adjoint_backward(pd_ctx* ctx, const double* lam_U, const double* lam_V, double* grad_f);

#ifdef __cplusplus
}
#endif
#endif
