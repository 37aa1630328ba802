// Internal declarations shared by the translation units of libpdmtel_b200.
//
// Device layout (HBM): every per-node vector is structure-of-arrays [3][N]
// (component-major) so that a warp of consecutive nodes reads 256 B per
// component; Gauss-point data are [npt*3][N]; the family is CSR with int64
// row offsets and int32 columns in ascending id order.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/pdmtel_b200.h"

namespace pd {

constexpr int kMaxPoints = 512;  // 8x8x8 Gauss rule

struct MatDev {
    double spring, density, ecrit, grav[3];
};

struct BcDev {
    int type;
    int dir[3];
    double val[9];
    double end_time;
    double load_type;
};

// Per-Gauss-point constants computed on the host in the reference's order:
// hg = (0.5*dx)*abscissa, W = ((vol8*w1)*w2)*w3, dxe = (effW*dx)/2,
// pw3 = pow(0.5*effW, 3) (pdDataManager.cpp:1932-1955, pdDataManager2.cpp:1313-1342).
struct GaussConst {
    double hg[3];
    double W;
    double dxe;
    double pw3;
    float hgf[3];
    float Wf;
    float A, B;  // beta = saturate((A - r) * B), FP32 form
};

// Everything a kernel needs, passed by value.
struct Dev {
    int64_t n;
    int npt;
    int cci, cci_mdf, mls, energy;
    double dx, delta, damping, vol, vol_cci;  // vol = pow(dx,3.0), vol_cci = (dx*dx)*dx
    const double* x;          // [3][N]
    const int32_t* mat;       // [N]
    const int32_t* bc;        // [N]
    const MatDev* mats;
    int nmat;
    const BcDev* bcs;
    int nbc;
    const double* bdry;       // [N]
    const double* sfac;       // [N] or nullptr
    const GaussConst* gc;     // [npt]
    const GaussConst* gc_host;  // host copy of gc (kernel-parameter constants)
    // family (full) and active (unbroken) CSR
    const int64_t* frow;
    const int32_t* fcol;
    const uint8_t* fbroken;
    const int64_t* arow;
    const int32_t* acol;
    // MLS, coefficient layout [node][contributor][point]
    const int64_t* cbptr;
    const int32_t* cbidx;
    const double* coeff;
    const float* coeff32;
    const float* csum;        // [N][npt] partition-of-unity defect sum(c)-1
    // state [3][N]
    double* U;
    double* V;
    double* vbuf;
    double* u1;
    double* us;
    double* k1;
    double* k2;
    double* k32;
    double* ug;               // [npt*3][N]
    double* eed;              // [N]
    double* red;              // reduction scratch
    double* tdev;             // current time (device scalar; advanced on the device)
    // work order: node-parallel kernels take node order[tid], so that a block
    // covers a compact 3-D tile of the lattice (its neighbours then share L1)
    const int32_t* order;
    // FP32 form, per node (array-of-structures, 16-byte aligned):
    //  nblk [N][bs]: Gauss-point displacement relative to the node, component-
    //        major ([x:npt][y:npt][z:npt]), then the node's trial displacement
    //        split into FP32 hi and lo parts (hi[3], lo[3]); rewritten by every
    //        gather (or, for CCI, by the pack kernel); chunk-major when blk_cm
    //        is set (below)
    //  sblk [N][8]:  coordinates split hi[3], lo[3], boundary factor, spring factor
    float* nblk;
    int bs;
    const float* sblk;
    int multimat, hasfail;
    int bdry_on;              // some boundary factor differs from 1
    // lattice positions packed x | y << 11 | z << 22 (x, y < 2048, z < 1024)
    // when every node sits on one cubic lattice of spacing dx; else nullptr
    const int32_t* lat;
    float c0, e0;             // spring and critical stretch when there is one material
    int acc_stretch;          // FP64 force: extension as (2 xi.eta + eta.eta)/(p + r)
    int64_t f64_lanes_below;  // FGI FP64 force: eight lanes per node below this many nodes
    int gather_per_point;     // FP32 gather: one thread per (node, point) instead of per 4 points
    // lattice box of the packed positions and the position -> node id map
    // (-1: no node); the FP32 force stages tile_x x tile_y x tile_z tiles in
    // shared memory when tile_x > 0 (fam_radius: largest family offset)
    const int32_t* pos2id;
    int lat_nx, lat_ny, lat_nz;
    int fam_radius;
    int tile_x, tile_y, tile_z;
    int force_quad;           // FP32 force: four nodes per thread (lattice, one material, no failure)
    // FP32 gather in SELL layout (16 nodes per slice of the work order, 2x2x2 points)
    int sell_on;
    const int64_t* sell_off;  // [slices + 1] first contributor slot of each slice
    const int32_t* sell_idx;  // [slots][16]
    const float* sell_coef;   // [slots][16][8]
    // FP32 force on the lattice stencil (2x2x2 points, one material, nodes
    // that form complete box lattices: box b holds the nodes first_b ..
    // first_b + nx ny nz - 1 with node id = first_b + x + nx (y + ny z); one
    // box, or the specimens of a batch).  blk_cm: nblk is stored chunk-major,
    // float4 chunk c of node j at nblk + 4 (c N + j), so that a warp reading
    // chunk c of x-adjacent nodes reads contiguous memory.  Work unit: the
    // x-adjacent node pair (2 px, 2 px + 1) of a row; a block covers tw pairs
    // x (sten_by 16 / tw) rows x sten_bz layers of one box, tw = sten_tw(the
    // box's pairs per row).  Union list U2 = S u (S +
    // e_x) (S: every lattice offset of a family entry; sten_nu entries, in
    // ascending neighbour id for every box): .x offset of the neighbour from
    // node A of the pair in node ids (one box), .y .z .w its lattice offset
    // from A.  Masks [side][word][pair]: bit u of a side set when U2 entry u
    // is an unbroken bond of that node.  sten_box[b] = (nx, ny, nz, first
    // tile), sten_boxb[b] = (first node, first pair), boxes in node order.
    int blk_cm;
    int sten_nu, sten_nw, sten_by, sten_bz;
    int64_t sten_np;
    int sten_nbox;
    int64_t sten_ntiles;
    uint8_t* sten_wide;           // [sten_ntiles] 1: the series pass left this tile to the exact pass
    const int4* sten_box;
    const longlong2* sten_boxb;
    const int4* sten_u2;
    const float4* sten_tab;       // [2][sten_nu][4] geometry of the stencil force (k_sten_table)
    const uint32_t* sten_mask;    // FP32 gather from contributor patterns: node i's contributors are
    // i + gpat_off[gpat_ptr[p] ..] with p = gpat_id[i] (the same ids in the same
    // order as its CSR list; nodes whose lists are translates share a pattern)
    const int32_t* gpat_id;
    const int64_t* gpat_ptr;
    const int32_t* gpat_off;
    // adaptive-trapezoid (AI) integration (pd_ai.cu): the force of a bond is
    // the sum of its regions' nested trapezoid integrals (pd_ai_eval.h)
    int ai, ai_n, ai_mls;         // on, trapezoid index 1..3, MLS on
    int64_t ai_nent, ai_ntab;     // full-family entries, MLS table entries
    const int64_t* ai_rptr;       // [H+1] regions of each full-family entry
    const pd_ai_region* ai_reg;
    const int32_t* ai_row;        // [H] node i of full-family entry i -> j
    const int64_t* ai_mirror;     // [H] entry j -> i
    const int64_t* ai_tptr;       // [N+1] MLS table entries of each node
    const int64_t* ai_coff;       // [N] first coefficient of each node's table
    const int32_t* ai_tnode;      // [T] node of each table entry
    const double* ai_tcoef;       // [entry][contributor of the node]
    double* ai_u;                 // [T][3] displacement of each table entry (per stage)
    double* ai_F;                 // [H][3] bond force of the stage
    int32_t* ai_fail;             // [H] points past the critical stretch in the stage's evaluation
    uint8_t* ai_brk;              // [H] broken: an AI bond breaks for good
    int32_t* ai_dmg;              // [N] failed points of the step (pdNode's damaged-bond count)
    int* ai_err;                  // a table entry out of range was asked for
    const int64_t* ai_eptr;       // [H+1] per-point energy slots of each entry (its trapezoid points)
    double* ai_e;                 // energy term of every point of the stage
    const int32_t* ai_order;      // [H] entries in the bond kernel's work order
};

// kernel launchers (pd_exact.cu: compiled without FMA contraction)
void launch_force_f64(const Dev& d, double dts, cudaStream_t s);
void launch_gather_f64(const Dev& d, const double* us, cudaStream_t s);
void launch_epilogue(const Dev& d, int stage, double dts, double dt, cudaStream_t s);
void launch_advance_time(double* t, double dt, cudaStream_t s);
void launch_energy_reduce(const Dev& d, cudaStream_t s);
// InitIntegrationPoint on the device (k_mls_contrib, k_mls_coeff): contributor
// CSR and coefficients [node][contributor][point] from the family and the MLS
// coordinates xm [3][N]; cnt [N] is scratch, cbptr [N+1] is written; the
// other arrays are allocated through alloc(actx, bytes).  PD_ERR_SINGULAR
// with *bad_node on a singular moment matrix.
int mls_setup(const Dev& d, const double* xm, double rw, const double* absc, int n1, int64_t* cnt, int64_t* cbptr,
              int32_t** cbidx, double** coeff, float** coeff32, float** csum, int64_t* total, int64_t* bad_node,
              void* (*alloc)(void*, size_t), void* actx, cudaStream_t s);
// PostAFD on the device (k_afd_gauss, k_afd_items): Gauss-point displacements
// of the nodal U [3][N] into ug [npt*3][N], then per item (node i, source s,
// direction 1..3) the half-space bond-force sum into out [items][3]; bE [N]
// the boundary factors to use, absc / wts the 1-D Gauss rule (n1 points).
int afd_forces(const Dev& d, const double* U, const double* bE, double* ug, const double* absc, const double* wts,
               int n1, int64_t n_items, const int64_t* item_i, const int64_t* item_s, const int32_t* item_d,
               double* out, cudaStream_t s);
void launch_to_soa(const double* aos, double* soa, int64_t n, int comps, cudaStream_t s);
void launch_to_soa_changed(const double* aos, double* soa, int64_t n, int comps, int* changed, cudaStream_t s);
void launch_to_aos(const double* soa, double* aos, int64_t n, int comps, cudaStream_t s);
void launch_fill(double* p, double v, int64_t n, cudaStream_t s);

// bond search (pd_exact.cu)
struct SearchGrid {
    double lo[3];
    double h;
    int64_t nc[3];
};
int bond_search(const Dev& d, const SearchGrid& g, const int32_t* cell_rank, int64_t ncell, int nslit,
                const double* slits_dev, int64_t** frow, int32_t** fcol, uint8_t** fbroken, int64_t** arow,
                int32_t** acol, int64_t* nh, int64_t* nb, double* min_bond, cudaStream_t s);

// adaptive-trapezoid (AI) form (pd_ai.cu, compiled without FMA contraction):
// the MLS table gather of a stage and the force stage
void launch_ai_gather(const Dev& d, const double* us, cudaStream_t s);
void launch_ai_force(const Dev& d, double dts, cudaStream_t s);

// FP32 compensated form (pd_f32c.cu)
void launch_force_f32c(const Dev& d, double dts, cudaStream_t s);
void launch_gather_f32c(const Dev& d, const double* us, cudaStream_t s);
void launch_pack_cci_f32c(const Dev& d, cudaStream_t s);
size_t tiled_smem_bytes(const Dev& d);
int64_t sell_slices(const Dev& d);
void launch_sell_width(const Dev& d, int64_t* width, cudaStream_t s);
void launch_sell_fill(const Dev& d, const int64_t* off, int32_t* sidx, float* scoef, cudaStream_t s);
int prepare_tiled_force(size_t smem);
void launch_family_radius(const Dev& d, int* out, cudaStream_t s);
// lattice-stencil force setup: offsets present in the families (bitmap over
// [-R, R]^3, R the family radius), the masks of every pair (err: set when a
// family does not fit the union list or a node breaks the box numbering)
void launch_sten_offsets(const Dev& d, int R, int* bitmap, int* err, cudaStream_t s);
void launch_sten_masks(const Dev& d, const int* lut, int R, uint32_t* mask, int* err, cudaStream_t s);
// geometry table of the stencil force (d.sten_u2, d.sten_nu, the Gauss
// constants) into tab [2][nu][4]; sets the kernel's shared-memory limit
int launch_sten_table(const Dev& d, float4* tab, cudaStream_t s);
// persistent FP32C stepping (pd_f32c.cu): control block of one launch.
// next[8*step + 2*(stage-1) + phase] are the work-queue counters; all of it
// is zeroed before every launch.
struct PersistCtl {
    unsigned arrive;
    int error;
    unsigned pad[30];
    unsigned next[1];  // [8 * nsteps]
};
// how long a grid barrier waits (ns) before giving up; stall: block 0 skips
// the first barrier (tests of the give-up path)
struct PersistWait {
    unsigned long long ns;
    int stall;
};
int persist_max_blocks(const Dev& d, int* per_sm, int* sms);
cudaError_t launch_persist_f32c(const Dev& d, double dt, int nsteps, PersistCtl* ctl, int blocks,
                                unsigned force_chunk, unsigned gather_chunk, PersistWait W, cudaStream_t s);

// CG helpers (pd_fast.cu): slots of the device scalar array
enum { CG_RR = 0, CG_PQ = 1, CG_RRN = 2, CG_BB = 3, CG_RES = 4, CG_NSLOT = 8 };
void launch_dot_f64(const double* a, const double* b, int64_t n, double* part, double* out, cudaStream_t s);
void launch_cg_update_x_f64(double* x, double* r, const double* p, const double* q, int64_t n, const double* scal, cudaStream_t s);
void launch_cg_update_p_f64(const double* r, double* p, int64_t n, const double* scal, cudaStream_t s);
void launch_cg_swap(double* scal, cudaStream_t s);
void launch_sub_f64(const double* a, const double* b, double* out, int64_t n, cudaStream_t s);
constexpr int kDotBlocks = 296;

// static operator (pd_fast.cu)
void launch_static_apply_f64(const Dev& d, double t, const double* x, double* y, cudaStream_t s);
// block-Jacobi preconditioner of the static operator ([6][N] symmetric
// inverses of the 3x3 diagonal blocks) and its application z = M^-1 r
void launch_static_bjacobi(const Dev& d, double* minv, cudaStream_t s);
void launch_bj_apply(const double* minv, const double* r, double* z, int64_t n, cudaStream_t s);
void launch_static_rhs(const Dev& d, double t, double* b, cudaStream_t s);
void launch_static_apply_f32x(const Dev& d, double t, const double* x, double* y, cudaStream_t s);
// the static operator on a complete box lattice (node id = x + nx (y + ny z))
// whose families are the horizon stencil clipped to the box
constexpr int kMaxStencil = 768;  // 64 B of shared memory each: under the 48 KB default
// Pairs per tile row of the stencil force for a box row of npx pairs: the
// widest of 16, 8, 4 whose padded row is within 1/8 of the least padded one
// (narrow boxes waste fewer lanes; wide ones keep 16).
__host__ __device__ inline int sten_tw(int npx) {
    const int p16 = (npx + 15) / 16 * 16, p8 = (npx + 7) / 8 * 8, p4 = (npx + 3) / 4 * 4;
    const int lim = p4 + p4 / 8;  // p4 is the least padded
    return p16 <= lim ? 16 : (p8 <= lim ? 8 : 4);
}

// Whether a box of npx pairs x ny rows x nz layers takes its stencil-force
// tiles as runs of 128 consecutive pairs in (x, y, z) order instead of 3D
// tiles of tw x by x bz: when the 3D tiles would leave more than a tenth of
// the lanes past the box (small specimens of a batch).
__host__ __device__ inline bool sten_linear(int npx, int ny, int nz, int tw, int by, int bz) {
    const long long np = (long long)npx * ny * nz;
    const long long pad =
        (long long)((npx + tw - 1) / tw * tw) * ((ny + by - 1) / by * by) * (long long)((nz + bz - 1) / bz * bz);
    return np * 10 < pad * 9;
}

struct StencilDev {
    int nx, ny, nz, ns;
    int radius;            // largest |offset| component
    const int4* off;       // [ns] lattice offset and node-id offset, ascending id offset
    const double4* geo;    // [ns] xi = offset * spacing, c V / r^3 of the one material
    const uint8_t* pmask;  // [N] prescribed directions, bits 0..2
    double* xm;            // [3N] scratch: the masked input (FP64, or FP32 in its first half)
    // the stencil regrouped into (ox, oy) columns: col[c] = (ox, oy, ox + nx oy,
    // 0) and colgeo[c][oz + rz] for oz in [-rz, rz] (c V / r^3 = 0 where the
    // offset is not in the stencil); ncol = 0 when rz is beyond 4
    int ncol, rz;
    const int4* col;
    const double4* colgeo;
    // the split form (k_static_nd): columns (ox, oy, ox + nx oy, h) sorted by
    // h, ndcls[h] .. ndcls[h + 1] - 1 the columns of half-height h; ndtap[c][oz
    // + 4] = (w, w oz sp); ndiag [6][N] the per-node diagonal blocks, ndint
    // the block of every node at least (nrx, nry, rz) inside the box (when
    // ndin: the box has such nodes); ndr the
    // nodes per thread along z (0: the difference form runs instead)
    int ndcol, ndr, nrx, nry, ndin;
    int ndcls[6];
    double sp;
    double ndint[6];
    const int4* ndc;
    const double2* ndtap;
    const double* ndiag;
    const struct NdTab* ndhost;  // host copy of the tables, passed as a kernel parameter
};
// The split form's tables as one kernel parameter (constant bank: warp-uniform
// reads through the constant cache, no shared-memory traffic).
constexpr int kNdMaxCol = 64;
struct NdTab {
    double2 tap[kNdMaxCol * 9];
    int4 col[kNdMaxCol];
};
void launch_static_pmask(const Dev& d, uint8_t* pm, cudaStream_t s);
void launch_static_stencil(const Dev& d, const StencilDev& S, bool f32, const double* x, double* y, cudaStream_t s);
void launch_static_ndiag(const StencilDev& S, int64_t n, double* D, cudaStream_t s);
size_t static_nd_smem(const StencilDev& S, int R);  // shared memory of the split-form kernel

// adjoint (pd_adjoint.cu): per-node adjoint vectors [3][N] of one RK4 step
struct AdjBuf {
    double *lU, *lV, *lvb, *lu1, *lk1, *lk2, *lk3, *lk4, *lus, *lF, *lueff;
};
void launch_vjp_own(const Dev& d, const double* teU, const double* teus, const double* teug, const double* lamF,
                    double* lam_u, double* gradf, cudaStream_t s, bool f32);
void launch_vjp_partner(const Dev& d, const double* teU, const double* teus, const double* teug, const double* lamF,
                        double* lam_ug, double* gradf, cudaStream_t s, bool f32);
// FP64 Gauss-point displacements [3 npt][N] from the FP32 form's node blocks
// (the node's trial displacement hi + lo plus each point's FP32 offset)
void launch_blocks_to_ug(const Dev& d, double* ug, cudaStream_t s);
void launch_gather_T(const Dev& d, const int64_t* tptr, const int32_t* tj, const int32_t* tpos, const double* lam_ug,
                     double* lam_us, cudaStream_t s);
void launch_adj_combine(const Dev& d, double dt, const double* lUp, const double* lVp, const AdjBuf& A,
                        cudaStream_t s);
void launch_adj_stage_pre(const Dev& d, double dts, const double* lk, const AdjBuf& A, cudaStream_t s);
void launch_adj_stage_node(const Dev& d, const AdjBuf& A, cudaStream_t s);
void launch_adj_stage_post(const Dev& d, double alpha, double* lk_prev, const AdjBuf& A, cudaStream_t s);
void launch_adj_stage1_end(const Dev& d, const AdjBuf& A, cudaStream_t s);

// scans and reductions (pd_fast.cu)
int exclusive_scan_i64(const int64_t* in, int64_t* out, int64_t n, cudaStream_t s);  // out has n+1 entries

}  // namespace pd

#define PD_CUDA_TRY(expr)                                                        \
    do {                                                                         \
        cudaError_t _e = (expr);                                                 \
        if (_e != cudaSuccess) return pd::fail_cuda(_e, #expr, __FILE__, __LINE__); \
    } while (0)

namespace pd {
int fail_cuda(cudaError_t e, const char* what, const char* file, int line);
int fail(int code, const char* msg);
}  // namespace pd
