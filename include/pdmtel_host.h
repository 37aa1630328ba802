/*
 * pdmtel_host.h — C ABI of the deck-level host layer (libpdmtel_b200.so).
 *
 * These entry points drive the C++ pdDataManager / pdSolve mirror of the
 * reference (pdDataManager.h:39-268, pdSolve.h:18-47) from C, ctypes or a
 * CLI: a working folder with pds_input.txt goes in, the reference's
 * InitialProblem / SolveDynamic / SolveStatic run on the GPU through
 * pdmtel_b200.h.  Status codes are the PD_ERR_* values of pdmtel_b200.h.
 */
#ifndef PDMTEL_HOST_H
#define PDMTEL_HOST_H

#include <stdint.h>

#include "pdmtel_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pdh_model pdh_model;

typedef struct pdh_info {
    int64_t num_nodes;
    int64_t num_halves;       /* family entries (2 x bonds) */
    int64_t num_broken;       /* family entries deleted by slits */
    int64_t num_contrib;      /* MLS contributor entries */
    int32_t num_gauss;        /* Gauss points per node */
    int32_t cci, mls, bdry_eff_on;
    int32_t dims[3];
    int32_t total_step, dump_frequency, num_max_family;
    double grid_spacing, horizon, total_time, stable_dt, min_bond_length;
    double ke, ee;            /* energies of the last RK4 step */
    int32_t num_materials, num_bcs, intg_point, pad;
    double damping;
} pdh_info;

/* SetWkDir + ReadInputFile (pdDataManager.cpp:4-758): dir holds pds_input.txt */
int pdh_open(const char* dir, pdh_model** out);
int pdh_close(pdh_model* m);
const char* pdh_last_error(pdh_model* m);
int pdh_get_info(pdh_model* m, pdh_info* info);

/* Batching (no counterpart in the reference): one model over `count`
 * specimen models opened with pdh_open (decks read; InitNode and
 * InitMaterial run here when not yet).  The specimens are placed side by side
 * on one lattice with gaps wider than the horizon, so pdh_init_bond finds no
 * bond between them, and pdh_init_integration_point solves each specimen's
 * MLS in its own coordinates.  Node ids run specimen by specimen
 * (pdh_batch_offsets, count + 1 entries).  Spring factors set on a specimen
 * (pdh_set_spring_factor) carry over.  All specimens must share the grid
 * spacing, horizon, integration scheme and damping, without boundary effect
 * factors.  out_dir receives the batch's log; the specimen models stay the
 * caller's.  Then continue as for one model: pdh_init_bond,
 * pdh_init_integration_point, pdh_context, the solve entry points. */
int pdh_batch_create(const char* out_dir, pdh_model* const* specimens, int count, pdh_model** out);
int pdh_batch_offsets(pdh_model* m, int64_t* offsets);
int pdh_batch_count(pdh_model* m, int* count);

/* the steps of pdSolve::InitialProblem (pdSolve.cpp:10-22) */
int pdh_init_node(pdh_model* m);
int pdh_init_bond(pdh_model* m);                 /* GPU */
int pdh_init_material(pdh_model* m);
int pdh_init_bdry_effect_factor(pdh_model* m);
int pdh_init_grid_boundary(pdh_model* m);
int pdh_init_integration_point(pdh_model* m);
int pdh_initial_problem(pdh_model* m);           /* all of the above */
/* installs a family CSR instead of pdh_init_bond (no GPU needed) */
int pdh_set_family(pdh_model* m, const int64_t* row_ptr, const int32_t* col, const uint8_t* broken, double min_bond);
/* per-node micromodulus factor (multiplies min(c_i,c_j) by (f_i+f_j)/2);
 * must precede the first GPU call */
int pdh_set_spring_factor(pdh_model* m, const double* f);

/* host copies of the setup arrays (sizes from pdh_get_info) */
int pdh_get_nodes(pdh_model* m, double* coords, int32_t* mat, int32_t* bc);
int pdh_get_family(pdh_model* m, int64_t* row_ptr, int32_t* col, uint8_t* broken);
int pdh_get_bdry_eff(pdh_model* m, double* bE);
int pdh_get_mls(pdh_model* m, int64_t* cb_ptr, int32_t* cb_idx, double* coeff);
/* the tables the device context is built from: materials (spring constant as
 * InitMaterial sets it, pdDataManager.cpp:1310-1322), boundary conditions,
 * and the 1-D Gauss rule (intg_point abscissae and weights) */
int pdh_get_tables(pdh_model* m, pd_material* materials, pd_bc* bcs, double* abscissae, double* weights);

/* the device context of the model (uploads the setup on first use) */
int pdh_context(pdh_model* m, pd_ctx** ctx);
int pdh_set_precision(pdh_model* m, int precision);
/* InitIntegrationPoint (pdDataManager2.cpp:106-309) on the device
 * (pd_mls_setup) when on != 0; set before InitIntegrationPoint.  Off by
 * default: the host setup reproduces the reference bit for bit. */
int pdh_set_device_setup(pdh_model* m, int on);
/* pdSolve::PostAFD (pdSolve.cpp:810-834) without the console: reads
 * pds_tecplot_<step>.dat of the working folder and writes the areal force
 * density stress of n requests to pds_AFD_<step>.dat; request k is a plane
 * (kind 1: nodes whose coordinate along norm[k] equals coord[k]) or a node
 * (kind 2: node[k]). */
int pdh_post_afd(pdh_model* m, int step, int n, const int32_t* kind, const int32_t* norm, const double* coord,
                 const int64_t* node);

/* pdSolve::SolveDynamic (pdSolve.cpp:24-130); write_files selects the
 * reference's per-step log, probe and Tecplot output */
int pdh_solve_dynamic(pdh_model* m, int write_files);
/* static solve of the linearised operator; the displacement becomes the
 * node state */
int pdh_solve_static(pdh_model* m, int precision, double rtol, int* iters, double* relres);

#ifdef __cplusplus
}
#endif
#endif
