// The C ABI of libpdmtel_b200 (include/pdmtel_b200.h): context life cycle,
// uploads in the reference's row layout, the RK4 driver and the static CG.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "pd_ai_eval.h"
#include "pd_internal.cuh"

namespace pd {

namespace {
thread_local std::string g_last_error;
}

int fail(int code, const char* msg) {
    g_last_error = msg ? msg : "";
    return code;
}

int fail_cuda(cudaError_t e, const char* what, const char* file, int line) {
    char buf[512];
    std::snprintf(buf, sizeof buf, "%s:%d %s: %s", file, line, what, cudaGetErrorString(e));
    g_last_error = buf;
    return e == cudaErrorMemoryAllocation ? PD_ERR_OOM : PD_ERR_CUDA;
}

}  // namespace pd

using pd::fail;

struct pd_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaStream_t copy_stream = nullptr;  // pd_rk4_steps_host: result copies beside the closing gather
    cudaEvent_t ev_final = nullptr, ev_copied = nullptr;
    pd::Dev d{};
    int64_t n = 0, H = 0, Ha = 0;
    int npt = 1;
    int precision = PD_PREC_FP64;
    int nslit = 0;
    std::vector<double> coords;  // [N][3] host copy
    std::vector<double> abscis;  // 1-D Gauss abscissae and weights (FGI)
    std::vector<double> gweights;
    std::vector<double> slits;
    double* dslits = nullptr;   // [nslit][6] on the device
    std::vector<pd::GaussConst> gch;            // Gauss constants (host copy)
    std::vector<double> bdry_host, sfac_host;   // per-node factors (host copies)
    std::vector<int32_t> bc_host;               // per-node bc index
    std::vector<int64_t> cbptr_host;            // MLS contributor CSR (host copy)
    std::vector<int32_t> cbidx_host;
    // adjoint: checkpoints (U, V, Gauss-point u, time) of the last forward
    struct Checkpoint {
        double *U = nullptr, *V = nullptr, *ug = nullptr;
        float* blk = nullptr;  // the FP32 form's node blocks (FP32C forward runs)
        double t = 0.0;
    };
    std::vector<Checkpoint> ckpt;
    int adj_steps = 0, adj_every = 0, adj_acc = 0;
    bool adj_f32 = false;  // the last forward run was the FP32-compensated form
    int adj_vjp32 = 0;     // PD_OPT_ADJOINT_VJP32: FP32 point terms in its reverse sweep
    // launch shapes (pd_set_option / pd_autotune)
    int64_t tile = 3 | (2 << 8) | (2 << 16);
    int persist_per_sm = 0;  // 0: as many as fit
    unsigned force_chunk = 128, gather_chunk = 256;
    // persistent stepping: control block and the graph of one launch
    pd::PersistCtl* pctl = nullptr;
    int pctl_steps = 0;
    cudaGraphExec_t persist_graph = nullptr;
    double persist_dt = 0.0, persist_t0 = 0.0;
    int persist_steps = 0;
    uint64_t persist_generation = ~0ull;
    int tuned_persistent = 0;
    int64_t persist_wait_us = 4000000;  // grid-barrier wait limit
    int persist_stall = 0;
    // static operator: per-material springs, lattice stencil (static_prepare)
    std::vector<double> mat_spring;
    int static_stencil_opt = 1;
    int static_precond = 1;        // block-Jacobi preconditioner of the static CG (PD_OPT_STATIC_PRECOND)
    double* bj_minv = nullptr;
    uint64_t bj_gen = ~0ull;
    int static_replacements = 0;
    bool sten_ok = false;
    uint64_t sten_gen = ~0ull;
    pd::StencilDev sten{};
    int4* sten_off = nullptr;
    double4* sten_geo = nullptr;
    uint8_t* sten_pmask = nullptr;
    double* sten_xm = nullptr;
    int4* sten_col = nullptr;
    double4* sten_colgeo = nullptr;
    int static_split = 4;           // split-form nodes per thread (PD_OPT_STATIC_SPLIT; 0: difference form)
    int64_t static_f32_below = 10;  // FP32 matvecs below relative residual 1/value (PD_OPT_STATIC_F32_BELOW)
    int4* nd_col = nullptr;
    double2* nd_tap = nullptr;
    double* nd_diag = nullptr;
    std::unique_ptr<pd::NdTab> nd_host;
    double adj_dt = 0.0;
    int64_t *tptr = nullptr;
    int32_t *tj = nullptr, *tpos = nullptr;
    int gpat_opt = 0;             // FP32 gather from contributor patterns (PD_OPT_GATHER_STENCIL)
    bool have_gpat = false;       // patterns built (with the MLS data; refused when nothing repeats)
    int32_t* gpat_id = nullptr;
    int64_t* gpat_ptr = nullptr;
    int32_t* gpat_off = nullptr;
    int fst_shape = 0;            // lattice-stencil FP32 force (PD_OPT_FORCE_STENCIL)
    int4* fst_u2 = nullptr;
    uint32_t* fst_mask = nullptr;
    float4* fst_tab = nullptr;
    uint8_t* fst_wide = nullptr;     // stencil force: tiles left to the exact pass (one byte per tile)
    int4* fst_box = nullptr;         // stencil force boxes (dims, first tile) and (first node, first pair)
    longlong2* fst_boxb = nullptr;
    std::vector<int64_t> box_first;  // pd_set_boxes: node ranges that are complete box lattices
    std::vector<int4> box_dims;
    int64_t* sell_off = nullptr;  // SELL copy of the FP32 gather's lists
    int32_t* sell_idx = nullptr;
    float* sell_coef = nullptr;
    double* adj_pool = nullptr;  // reverse-sweep work buffers and stage tape
    int64_t adj_pool_count = 0;
    bool have_family = false, have_mls = false;
    bool have_ai = false;                   // pd_set_ai data for the current family
    int64_t ai_points = 0;                  // trapezoid points of the unbroken bonds per stage
    std::vector<void*> ai_bufs;             // device buffers of the AI form
    std::vector<int32_t> bctype_host;       // per bc: its type
    // owned device buffers
    std::vector<void*> owned;
    int64_t *frow = nullptr, *arow = nullptr, *cbptr = nullptr;
    int32_t *fcol = nullptr, *acol = nullptr, *cbidx = nullptr;
    uint8_t* fbroken = nullptr;
    double *coeff = nullptr, *scratch = nullptr, *dotpart = nullptr, *scal = nullptr;
    float *coeff32 = nullptr, *csum = nullptr;
    double* hstage = nullptr;  // pinned host staging, 3N doubles x 2
    double* hscalar = nullptr; // pinned host scalars
    int* dflag = nullptr;      // device flags (pd_rk4_steps_host: the uploaded U differs)
    // CUDA graph of one RK4 step
    cudaGraphExec_t step_graph = nullptr;
    double graph_dt = 0.0;
    int graph_prec = -1, graph_energy = -1;
    uint64_t generation = 0, graph_generation = ~0ull;
};

namespace {

template <typename T>
int dalloc(pd_ctx* c, T** p, size_t count) {
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T));
    if (e != cudaSuccess) return pd::fail_cuda(e, "cudaMalloc", __FILE__, __LINE__);
    c->owned.push_back(q);
    *p = (T*)q;
    return PD_OK;
}

void dfree(pd_ctx* c, void* p) {
    if (!p) return;
    auto it = std::find(c->owned.begin(), c->owned.end(), p);
    if (it != c->owned.end()) c->owned.erase(it);
    cudaFree(p);
}

#define PD_TRY(expr)                       \
    do {                                   \
        int _rc = (expr);                  \
        if (_rc != PD_OK) return _rc;      \
    } while (0)

int upload(pd_ctx* c, void* dst, const void* src, size_t bytes) {
    PD_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->stream));
    PD_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return PD_OK;
}

// [N][3] host -> [3][N] device (through the scratch buffer)
int upload_vec3(pd_ctx* c, double* dst_soa, const double* src_aos) {
    if (c->n == 0) return PD_OK;
    const size_t bytes = sizeof(double) * 3 * c->n;
    std::memcpy(c->hstage, src_aos, bytes);
    PD_CUDA_TRY(cudaMemcpyAsync(c->scratch, c->hstage, bytes, cudaMemcpyHostToDevice, c->stream));
    pd::launch_to_soa(c->scratch, dst_soa, c->n, 3, c->stream);
    PD_CUDA_TRY(cudaGetLastError());
    PD_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return PD_OK;
}

int download_vec3(pd_ctx* c, double* dst_aos, const double* src_soa) {
    if (c->n == 0) return PD_OK;
    const size_t bytes = sizeof(double) * 3 * c->n;
    pd::launch_to_aos(src_soa, c->scratch, c->n, 3, c->stream);
    PD_CUDA_TRY(cudaGetLastError());
    PD_CUDA_TRY(cudaMemcpyAsync(c->hstage, c->scratch, bytes, cudaMemcpyDeviceToHost, c->stream));
    PD_CUDA_TRY(cudaStreamSynchronize(c->stream));
    std::memcpy(dst_aos, c->hstage, bytes);
    return PD_OK;
}

int set_time(pd_ctx* c, double t) {
    *c->hscalar = t;
    PD_CUDA_TRY(cudaMemcpyAsync(c->d.tdev, c->hscalar, sizeof(double), cudaMemcpyHostToDevice, c->stream));
    PD_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return PD_OK;
}

// Static per-node block of the FP32 form: coordinates split hi/lo, boundary
// factor, spring factor.
int upload_static_f32(pd_ctx* c) {
    const int64_t N = c->n;
    std::vector<float> h((size_t)N * 8);
    for (int64_t i = 0; i < N; ++i) {
        float* o = &h[8 * i];
        for (int a = 0; a < 3; ++a) {
            const double x = c->coords[3 * i + a];
            o[a] = (float)x;
            o[3 + a] = (float)(x - (double)o[a]);
        }
        o[6] = (float)c->bdry_host[i];
        o[7] = c->sfac_host.empty() ? 1.0f : (float)c->sfac_host[i];
    }
    return upload(c, (void*)c->d.sblk, h.data(), sizeof(float) * h.size());
}

// Work order of the node-parallel kernels: nodes grouped into 8x4x4 tiles of
// lattice positions (x fastest inside a tile), tiles in x, y, z order, so
// that a 128-thread block covers one compact tile.
// Work order: lattice tiles of 2^bx x 2^by x 2^bz nodes, tiles in x-fastest
// order, nodes x-fastest inside a tile (x-adjacent nodes pair up in the
// FP32 pair kernel).  Default 8 x 4 x 4.
std::vector<int32_t> tiled_order(const std::vector<double>& x, int64_t N, double dx, int bx = 3, int by = 2,
                                 int bz = 2) {
    std::vector<int32_t> ord(N);
    if (N == 0) return ord;
    double lo[3] = {x[0], x[1], x[2]};
    for (int64_t i = 0; i < N; ++i)
        for (int a = 0; a < 3; ++a) lo[a] = std::min(lo[a], x[3 * i + a]);
    std::vector<std::pair<uint64_t, int32_t>> key(N);
    const int lb = bx + by + bz;
    for (int64_t i = 0; i < N; ++i) {
        int64_t l[3];
        for (int a = 0; a < 3; ++a) l[a] = (int64_t)std::llround((x[3 * i + a] - lo[a]) / dx);
        const uint64_t tx = l[0] >> bx, ty = l[1] >> by, tz = l[2] >> bz;
        const uint64_t tile = (tz << 38) | (ty << 19) | tx;
        const uint64_t local = ((uint64_t)(l[2] & ((1 << bz) - 1)) << (bx + by)) |
                               ((uint64_t)(l[1] & ((1 << by) - 1)) << bx) | (uint64_t)(l[0] & ((1 << bx) - 1));
        key[i] = {(tile << lb) | local, (int32_t)i};
    }
    std::sort(key.begin(), key.end());
    for (int64_t k = 0; k < N; ++k) ord[k] = key[k].second;
    return ord;
}

// Packed lattice positions x | y << 11 | z << 22 when every node lies within
// 1e-6 spacings of the cubic lattice through the lowest corner (the lattices
// InitNode generates, pdDataManager.cpp:846-907); false otherwise.
bool lattice_positions(const std::vector<double>& x, int64_t N, double dx, std::vector<int32_t>& out) {
    if (N == 0) return false;
    double lo[3] = {x[0], x[1], x[2]};
    for (int64_t i = 0; i < N; ++i)
        for (int a = 0; a < 3; ++a) lo[a] = std::min(lo[a], x[3 * i + a]);
    const int64_t lim[3] = {2048, 2048, 1024};
    out.assign(N, 0);
    for (int64_t i = 0; i < N; ++i) {
        int64_t l[3];
        for (int a = 0; a < 3; ++a) {
            l[a] = (int64_t)std::llround((x[3 * i + a] - lo[a]) / dx);
            if (l[a] < 0 || l[a] >= lim[a]) return false;
            if (std::fabs(x[3 * i + a] - (lo[a] + (double)l[a] * dx)) > 1e-6 * dx) return false;
        }
        out[i] = (int32_t)(l[0] | (l[1] << 11) | (l[2] << 22));
    }
    return true;
}

uint64_t morton3(uint64_t x, uint64_t y, uint64_t z) {
    auto spread = [](uint64_t v) {
        v &= 0x1fffff;
        v = (v | v << 32) & 0x1f00000000ffffull;
        v = (v | v << 16) & 0x1f0000ff0000ffull;
        v = (v | v << 8) & 0x100f00f00f00f00full;
        v = (v | v << 4) & 0x10c30c30c30c30c3ull;
        v = (v | v << 2) & 0x1249249249249249ull;
        return v;
    };
    return spread(x) | spread(y) << 1 | spread(z) << 2;
}

bool ready_dynamic(pd_ctx* c) {
    if (!c->have_family) return false;
    if (c->d.ai) return c->have_ai;
    if (!c->d.cci && c->d.mls && !c->have_mls) return false;
    return true;
}

// the four stages of pdDataManager::RK4 and the closing gather
void enqueue_step_body(pd_ctx* c, double dt, bool closing_gather = true) {
    cudaStream_t s = c->stream;
    const pd::Dev& d = c->d;
    const int64_t n3 = 3 * c->n;
    const bool f32 = c->precision == PD_PREC_FP32C;
    auto force = [&](double dts) {
        if (f32) pd::launch_force_f32c(d, dts, s);
        else pd::launch_force_f64(d, dts, s);
    };
    auto gather = [&](const double* us) {
        if (f32) pd::launch_gather_f32c(d, us, s);
        else pd::launch_gather_f64(d, us, s);
    };
    const double dtHalf = 0.5 * dt;
    // InitDynamicSolve: vbuf = V, energy density 0; u1 = us = U
    cudaMemcpyAsync(d.vbuf, d.V, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(d.u1, d.U, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(d.us, d.U, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s);
    if (d.energy) cudaMemsetAsync(d.eed, 0, sizeof(double) * c->n, s);
    if (d.ai) cudaMemsetAsync(d.ai_dmg, 0, sizeof(int32_t) * c->n, s);
    force(dtHalf);
    pd::launch_epilogue(d, 1, dtHalf, dt, s);
    gather(d.us);
    force(dtHalf);
    pd::launch_epilogue(d, 2, dtHalf, dt, s);
    gather(d.us);
    force(dt);
    pd::launch_epilogue(d, 3, dt, dt, s);
    gather(d.us);
    force(dt);
    pd::launch_epilogue(d, 4, dt, dt, s);
    if (d.energy) pd::launch_energy_reduce(d, s);
    if (closing_gather) gather(d.U);
}

// the closing gather of a step alone (CalcIntgPointDisplRK4 at the new U)
void enqueue_closing_gather(pd_ctx* c) {
    if (c->precision == PD_PREC_FP32C) pd::launch_gather_f32c(c->d, c->d.U, c->stream);
    else pd::launch_gather_f64(c->d, c->d.U, c->stream);
}

}  // namespace

extern "C" {

int pd_abi_version(void) { return PD_ABI_VERSION; }

const char* pd_last_error(void) { return pd::g_last_error.c_str(); }

int pd_device_count(int* count) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) n = 0;
    if (count) *count = n;
    return PD_OK;
}

int pd_ctx_create(const pd_problem* P, pd_ctx** out) {
    if (!P || !out) return fail(PD_ERR_ARG, "pd_ctx_create: null argument");
    *out = nullptr;
    if (P->num_nodes < 0 || (P->num_nodes > 0 && (!P->coords || !P->mat_id)))
        return fail(PD_ERR_ARG, "pd_ctx_create: bad node arrays");
    if (P->num_nodes > INT32_MAX) return fail(PD_ERR_ARG, "pd_ctx_create: more than 2^31-1 nodes");
    if (P->num_materials <= 0 || !P->materials) return fail(PD_ERR_ARG, "pd_ctx_create: no materials");
    if (P->num_bcs < 0 || (P->num_bcs > 0 && !P->bcs)) return fail(PD_ERR_ARG, "pd_ctx_create: bad bc table");
    if (!(P->grid_spacing > 0.0) || !(P->horizon > 0.0)) return fail(PD_ERR_ARG, "pd_ctx_create: bad spacing/horizon");
    if (P->integration != PD_INTG_CCI && P->integration != PD_INTG_FGI && P->integration != PD_INTG_AI)
        return fail(PD_ERR_ARG, "pd_ctx_create: unknown integration scheme");
    if (P->integration == PD_INTG_AI && (P->intg_point < 1 || P->intg_point > 3))
        return fail(PD_ERR_ARG, "pd_ctx_create: the AI trapezoid index must be 1..3 (above 3 the reference's rule "
                                "refines a sum left by the previous integral)");
    int n1 = P->integration == PD_INTG_FGI ? P->intg_point : 1;
    if (n1 < 1 || n1 > 8) return fail(PD_ERR_ARG, "pd_ctx_create: intg_point must be 1..8");
    if (P->integration == PD_INTG_FGI && (!P->abscissae || !P->weights))
        return fail(PD_ERR_ARG, "pd_ctx_create: Gauss abscissae/weights required");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(PD_ERR_NODEV, "no CUDA device");
    const int64_t N = P->num_nodes;
    for (int64_t i = 0; i < N; ++i) {
        if (P->mat_id[i] < 0 || P->mat_id[i] >= P->num_materials) return fail(PD_ERR_ARG, "mat_id out of range");
        if (P->bc_id && (P->bc_id[i] < -1 || P->bc_id[i] >= P->num_bcs)) return fail(PD_ERR_ARG, "bc_id out of range");
    }
    pd_ctx* c = new pd_ctx();
    auto bail = [&](int rc) {
        pd_ctx_destroy(c);
        return rc;
    };
    cudaGetDevice(&c->device);
    if (P->stream) {
        c->stream = (cudaStream_t)P->stream;
    } else {
        cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) return bail(pd::fail_cuda(e, "cudaStreamCreate", __FILE__, __LINE__));
        c->own_stream = true;
    }
    c->n = N;
    c->npt = n1 * n1 * n1;
    c->coords.assign(P->coords, P->coords + 3 * N);
    if (P->integration == PD_INTG_FGI && P->abscissae) c->abscis.assign(P->abscissae, P->abscissae + n1);
    if (P->integration == PD_INTG_FGI && P->weights) c->gweights.assign(P->weights, P->weights + n1);
    c->nslit = P->num_slits > 0 ? P->num_slits : 0;
    if (c->nslit) c->slits.assign(P->slits, P->slits + 6 * c->nslit);
    pd::Dev& d = c->d;
    d.n = N;
    d.npt = c->npt;
    d.cci = P->integration == PD_INTG_CCI;
    d.cci_mdf = P->cci_modified ? 1 : 0;
    d.mls = (P->integration == PD_INTG_FGI && n1 > 1) ? 1 : 0;
    d.ai = P->integration == PD_INTG_AI;
    d.ai_n = d.ai ? P->intg_point : 0;
    d.energy = 1;
    d.dx = P->grid_spacing;
    d.delta = P->horizon;
    d.damping = P->damping;
    d.vol = std::pow(d.dx, 3.0);           // node volume, pdDataManager.cpp:1081
    d.vol_cci = d.dx * d.dx * d.dx;        // pdDataManager2.cpp:1328
    const size_t n3 = (size_t)(3 * N);
    if (cudaMallocHost(&c->hstage, sizeof(double) * std::max<size_t>(n3, 1) * 2) != cudaSuccess)
        return bail(fail(PD_ERR_OOM, "pinned staging"));
    if (cudaMallocHost(&c->hscalar, sizeof(double) * 16) != cudaSuccess) return bail(fail(PD_ERR_OOM, "pinned scalar"));
    double* x = nullptr;
    int32_t *mat = nullptr, *bc = nullptr;
    pd::MatDev* mats = nullptr;
    pd::BcDev* bcs = nullptr;
    pd::GaussConst* gc = nullptr;
    double* bdry = nullptr;
    int rc = PD_OK;
    if ((rc = dalloc(c, &c->scratch, n3 * 2)) != PD_OK) return bail(rc);
    if ((rc = dalloc(c, &c->dflag, 4)) != PD_OK) return bail(rc);
    if ((rc = dalloc(c, &x, n3)) != PD_OK) return bail(rc);
    if ((rc = dalloc(c, &mat, N)) != PD_OK) return bail(rc);
    if ((rc = dalloc(c, &bc, N)) != PD_OK) return bail(rc);
    if ((rc = dalloc(c, &mats, P->num_materials)) != PD_OK) return bail(rc);
    if ((rc = dalloc(c, &bcs, std::max(P->num_bcs, 1))) != PD_OK) return bail(rc);
    if ((rc = dalloc(c, &gc, c->npt)) != PD_OK) return bail(rc);
    if ((rc = dalloc(c, &bdry, N)) != PD_OK) return bail(rc);
    double *U, *V, *vbuf, *u1, *us, *k1, *k2, *k32, *ug, *eed, *red, *tdev;
    float *nblk, *sblk;
    int32_t* order;
    d.bs = ((3 * c->npt + 6) + 3) / 4 * 4;
    if ((rc = dalloc(c, &U, n3)) || (rc = dalloc(c, &V, n3)) || (rc = dalloc(c, &vbuf, n3)) ||
        (rc = dalloc(c, &u1, n3)) || (rc = dalloc(c, &us, n3)) || (rc = dalloc(c, &k1, n3)) ||
        (rc = dalloc(c, &k2, n3)) || (rc = dalloc(c, &k32, n3)) || (rc = dalloc(c, &ug, n3 * c->npt)) ||
        (rc = dalloc(c, &nblk, (size_t)N * d.bs)) || (rc = dalloc(c, &sblk, (size_t)N * 8)) ||
        (rc = dalloc(c, &order, N)) || (rc = dalloc(c, &eed, N)) ||
        (rc = dalloc(c, &red, 2 * N + 4 + 2 * 160)) || (rc = dalloc(c, &tdev, 1)) ||
        (rc = dalloc(c, &c->dotpart, pd::kDotBlocks + 8)) || (rc = dalloc(c, &c->scal, pd::CG_NSLOT)))
        return bail(rc);
    if (c->nslit) {
        double* sl = nullptr;
        if ((rc = dalloc(c, &sl, 6 * c->nslit)) != PD_OK) return bail(rc);
        if ((rc = upload(c, sl, c->slits.data(), sizeof(double) * 6 * c->nslit)) != PD_OK) return bail(rc);
        c->dslits = sl;
    }
    // materials, boundary conditions, Gauss constants
    std::vector<pd::MatDev> hm(P->num_materials);
    for (int k = 0; k < P->num_materials; ++k) {
        hm[k].spring = P->materials[k].spring;
        hm[k].density = P->materials[k].density;
        hm[k].ecrit = P->materials[k].ecrit;
        for (int a = 0; a < 3; ++a) hm[k].grav[a] = P->materials[k].grav[a];
    }
    std::vector<pd::BcDev> hb(std::max(P->num_bcs, 1));
    for (int k = 0; k < P->num_bcs; ++k) {
        hb[k].type = P->bcs[k].type;
        for (int a = 0; a < 3; ++a) hb[k].dir[a] = P->bcs[k].dir[a];
        for (int a = 0; a < 9; ++a) hb[k].val[a] = P->bcs[k].value[a];
        hb[k].end_time = P->bcs[k].end_time;
        hb[k].load_type = P->bcs[k].load_type;
    }
    std::vector<pd::GaussConst> hg(c->npt);
    {
        const double vol8 = std::pow(d.dx, 3.0) / 8.0;  // pow(_gridSpacing, 3)/8.0, pdDataManager.cpp:1953
        std::vector<double> a(n1, 0.0), w(n1, 2.0);
        if (P->integration == PD_INTG_FGI) {
            for (int k = 0; k < n1; ++k) { a[k] = P->abscissae[k]; w[k] = P->weights[k]; }
        }
        for (int i = 0; i < n1; ++i)
            for (int j = 0; j < n1; ++j)
                for (int k = 0; k < n1; ++k) {
                    pd::GaussConst& G = hg[(i * n1 + j) * n1 + k];
                    G.hg[0] = 0.5 * d.dx * a[i];
                    G.hg[1] = 0.5 * d.dx * a[j];
                    G.hg[2] = 0.5 * d.dx * a[k];
                    const double w1 = w[i], w2 = w[j], w3 = w[k];
                    const double effw = std::pow(w1 * w2 * w3, 1.0 / 3.0);
                    G.W = vol8 * w1 * w2 * w3;
                    G.dxe = effw * d.dx / 2.0;
                    G.pw3 = std::pow(0.5 * effw, 3);
                    for (int q = 0; q < 3; ++q) G.hgf[q] = (float)G.hg[q];
                    G.Wf = (float)G.W;
                    G.A = (float)(d.delta + 0.5 * G.dxe);
                    G.B = (float)(1.0 / G.dxe);
                }
    }
    std::vector<double> xs(n3);
    for (int64_t i = 0; i < N; ++i)
        for (int a = 0; a < 3; ++a) xs[a * N + i] = P->coords[3 * i + a];
    std::vector<int32_t> bcv(N, -1);
    if (P->bc_id) std::copy(P->bc_id, P->bc_id + N, bcv.begin());
    c->bc_host = bcv;
    for (int k = 0; k < P->num_bcs; ++k) c->bctype_host.push_back(P->bcs[k].type);
    std::vector<double> ones(N, 1.0);
    if ((rc = upload(c, x, xs.data(), sizeof(double) * n3)) || (rc = upload(c, mat, P->mat_id, sizeof(int32_t) * N)) ||
        (rc = upload(c, bc, bcv.data(), sizeof(int32_t) * N)) ||
        (rc = upload(c, mats, hm.data(), sizeof(pd::MatDev) * hm.size())) ||
        (rc = upload(c, bcs, hb.data(), sizeof(pd::BcDev) * hb.size())) ||
        (rc = upload(c, gc, hg.data(), sizeof(pd::GaussConst) * hg.size())) ||
        (rc = upload(c, bdry, ones.data(), sizeof(double) * N)))
        return bail(rc);
    if (P->spring_factor) {
        double* sf = nullptr;
        if ((rc = dalloc(c, &sf, N)) != PD_OK || (rc = upload(c, sf, P->spring_factor, sizeof(double) * N)) != PD_OK)
            return bail(rc);
        d.sfac = sf;
        c->sfac_host.assign(P->spring_factor, P->spring_factor + N);
    }
    // FP32-form constants: one material -> kernel constants; a failure test
    // only when some critical stretch is within reach
    d.multimat = P->num_materials > 1;
    d.f64_lanes_below = int64_t(1) << 17;
    d.c0 = (float)P->materials[0].spring;
    d.e0 = (float)P->materials[0].ecrit;
    d.hasfail = 0;
    for (int k = 0; k < P->num_materials; ++k) d.hasfail |= !(P->materials[k].ecrit >= 1e10);
    c->gch = hg;
    d.gc_host = c->gch.data();
    c->bdry_host.assign(N, 1.0);
    for (int k = 0; k < P->num_materials; ++k) c->mat_spring.push_back(P->materials[k].spring);
    d.nblk = nblk;
    d.sblk = sblk;
    d.order = order;
    if ((rc = upload_static_f32(c)) != PD_OK) return bail(rc);
    {
        std::vector<int32_t> ord = tiled_order(c->coords, N, d.dx);
        if ((rc = upload(c, order, ord.data(), sizeof(int32_t) * N)) != PD_OK) return bail(rc);
        std::vector<int32_t> lat;
        if (lattice_positions(c->coords, N, d.dx, lat)) {
            int32_t* dl = nullptr;
            if ((rc = dalloc(c, &dl, N)) != PD_OK || (rc = upload(c, dl, lat.data(), sizeof(int32_t) * N)) != PD_OK)
                return bail(rc);
            d.lat = dl;
            // the lattice box and, when it is not much larger than the node
            // set, the position -> node id map of the tiled FP32 force
            int64_t nx = 0, ny = 0, nz = 0;
            for (int64_t i = 0; i < N; ++i) {
                nx = std::max<int64_t>(nx, (lat[i] & 2047) + 1);
                ny = std::max<int64_t>(ny, ((lat[i] >> 11) & 2047) + 1);
                nz = std::max<int64_t>(nz, (lat[i] >> 22) + 1);
            }
            d.lat_nx = (int)nx;
            d.lat_ny = (int)ny;
            d.lat_nz = (int)nz;
            if (nx * ny * nz <= 8 * N) {
                std::vector<int32_t> map((size_t)(nx * ny * nz), -1);
                for (int64_t i = 0; i < N; ++i)
                    map[(lat[i] & 2047) + nx * (((lat[i] >> 11) & 2047) + ny * (lat[i] >> 22))] = (int32_t)i;
                int32_t* dm = nullptr;
                if ((rc = dalloc(c, &dm, map.size())) != PD_OK ||
                    (rc = upload(c, dm, map.data(), sizeof(int32_t) * map.size())) != PD_OK)
                    return bail(rc);
                d.pos2id = dm;
            }
        }
    }
    d.x = x;
    d.mat = mat;
    d.bc = bc;
    d.mats = mats;
    d.nmat = P->num_materials;
    d.bcs = bcs;
    d.nbc = P->num_bcs;
    d.bdry = bdry;
    d.gc = gc;
    d.U = U;
    d.V = V;
    d.vbuf = vbuf;
    d.u1 = u1;
    d.us = us;
    d.k1 = k1;
    d.k2 = k2;
    d.k32 = k32;
    d.ug = ug;
    d.eed = eed;
    d.red = red;
    d.tdev = tdev;
    cudaMemsetAsync(U, 0, sizeof(double) * n3, c->stream);
    cudaMemsetAsync(V, 0, sizeof(double) * n3, c->stream);
    cudaMemsetAsync(vbuf, 0, sizeof(double) * n3, c->stream);
    cudaMemsetAsync(u1, 0, sizeof(double) * n3, c->stream);
    cudaMemsetAsync(us, 0, sizeof(double) * n3, c->stream);
    cudaMemsetAsync(ug, 0, sizeof(double) * n3 * c->npt, c->stream);
    cudaMemsetAsync(nblk, 0, sizeof(float) * N * d.bs, c->stream);
    cudaMemsetAsync(eed, 0, sizeof(double) * N, c->stream);
    cudaMemsetAsync(tdev, 0, sizeof(double), c->stream);
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return bail(pd::fail_cuda(e, "init", __FILE__, __LINE__));
    *out = c;
    return PD_OK;
}

int pd_ctx_destroy(pd_ctx* c) {
    if (!c) return PD_OK;
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->step_graph) cudaGraphExecDestroy(c->step_graph);
    if (c->persist_graph) cudaGraphExecDestroy(c->persist_graph);
    for (void* p : c->owned)
        if (p) cudaFree(p);
    if (c->hstage) cudaFreeHost(c->hstage);
    if (c->hscalar) cudaFreeHost(c->hscalar);
    if (c->copy_stream) {
        cudaStreamSynchronize(c->copy_stream);
        cudaStreamDestroy(c->copy_stream);
    }
    if (c->ev_final) cudaEventDestroy(c->ev_final);
    if (c->ev_copied) cudaEventDestroy(c->ev_copied);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return PD_OK;
}

int pd_ctx_stream(pd_ctx* c, void** s) {
    if (!c || !s) return fail(PD_ERR_ARG, "pd_ctx_stream: null argument");
    *s = (void*)c->stream;
    return PD_OK;
}

int pd_sync(pd_ctx* c) {
    if (!c) return fail(PD_ERR_ARG, "pd_sync: null context");
    PD_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return PD_OK;
}

// The SELL copy of the FP32 gather's contributor lists, in the current work
// order (rebuilt after pd_set_mls and after a work-order change; freed when
// the gather cannot use it).
static int sell_prepare(pd_ctx* c) {
    dfree(c, c->sell_off);
    dfree(c, c->sell_idx);
    dfree(c, c->sell_coef);
    c->sell_off = nullptr;
    c->sell_idx = nullptr;
    c->sell_coef = nullptr;
    c->d.sell_off = nullptr;
    c->d.sell_idx = nullptr;
    c->d.sell_coef = nullptr;
    if (!c->d.sell_on || !c->have_mls || !c->d.mls || c->npt != 8 || c->n == 0) return PD_OK;
    const int64_t S = pd::sell_slices(c->d);
    int64_t* width = nullptr;
    PD_TRY(dalloc(c, &width, S));
    PD_TRY(dalloc(c, &c->sell_off, S + 1));
    pd::launch_sell_width(c->d, width, c->stream);
    int rc = pd::exclusive_scan_i64(width, c->sell_off, S, c->stream);
    dfree(c, width);
    if (rc != PD_OK) return fail(PD_ERR_CUDA, "SELL layout: scan");
    int64_t total = 0;
    PD_CUDA_TRY(cudaMemcpy(&total, c->sell_off + S, sizeof(int64_t), cudaMemcpyDeviceToHost));
    PD_TRY(dalloc(c, &c->sell_idx, total * 16));
    PD_TRY(dalloc(c, &c->sell_coef, total * 16 * 8));
    c->d.sell_off = c->sell_off;
    c->d.sell_idx = c->sell_idx;
    c->d.sell_coef = c->sell_coef;
    pd::launch_sell_fill(c->d, c->sell_off, c->sell_idx, c->sell_coef, c->stream);
    PD_CUDA_TRY(cudaStreamSynchronize(c->stream));
    c->generation++;
    return PD_OK;
}

// The contributor patterns of the FP32 gather: every node's MLS contributor
// list as id offsets from the node, identical lists stored once (on a box
// lattice numbered x + nx (y + ny z) the lists of nodes with the same
// position relative to the boundary are translates of each other; in a
// batch, per specimen).  Built with the MLS data (pd_set_mls), whether or not
// a gather uses them.
static void gpat_free(pd_ctx* c) {
    for (void* p : {(void*)c->gpat_id, (void*)c->gpat_ptr, (void*)c->gpat_off}) dfree(c, p);
    c->gpat_id = nullptr;
    c->gpat_ptr = nullptr;
    c->gpat_off = nullptr;
    c->have_gpat = false;
    c->d.gpat_id = nullptr;
    c->d.gpat_ptr = nullptr;
    c->d.gpat_off = nullptr;
    c->generation++;
}

// the patterns are read by the gathers only while PD_OPT_GATHER_STENCIL is on
static void gpat_apply(pd_ctx* c) {
    const bool on = c->gpat_opt && c->have_gpat;
    c->d.gpat_id = on ? c->gpat_id : nullptr;
    c->d.gpat_ptr = on ? c->gpat_ptr : nullptr;
    c->d.gpat_off = on ? c->gpat_off : nullptr;
    c->generation++;
}

static int gpat_build(pd_ctx* c) {
    gpat_free(c);
    if (!c->have_mls || !c->d.mls || c->n == 0) return PD_OK;
    const int64_t N = c->n;
    const std::vector<int64_t>& cp = c->cbptr_host;
    const std::vector<int32_t>& ci = c->cbidx_host;
    std::vector<int32_t> pid((size_t)N);
    std::vector<int64_t> ptr{0};
    std::vector<int32_t> off;
    std::unordered_map<uint64_t, std::vector<int32_t>> seen;  // content hash -> pattern ids
    // refused when the distinct lists would hold more than a quarter of all
    // entries (little repeats: the table would not stay in cache), or above
    // 64M entries; at least 4M are allowed
    const size_t kMaxEntries =
        std::min<size_t>((size_t)64 << 20, std::max<size_t>((size_t)4 << 20, (size_t)cp[N] / 4));
    for (int64_t i = 0; i < N; ++i) {
        const int64_t b = cp[i], e = cp[i + 1];
        uint64_t h = 1469598103934665603ull ^ (uint64_t)(e - b);
        for (int64_t k = b; k < e; ++k) h = (h ^ (uint64_t)(uint32_t)(ci[k] - (int32_t)i)) * 1099511628211ull;
        auto& ids = seen[h];
        int32_t found = -1;
        for (int32_t q : ids) {
            const int64_t pb = ptr[q], pe = ptr[q + 1];
            if (pe - pb != e - b) continue;
            bool same = true;
            for (int64_t k = 0; k < e - b && same; ++k) same = off[pb + k] == ci[b + k] - (int32_t)i;
            if (same) {
                found = q;
                break;
            }
        }
        if (found < 0) {
            if (off.size() + (size_t)(e - b) > kMaxEntries) return PD_OK;  // the lists do not repeat
            found = (int32_t)(ptr.size() - 1);
            for (int64_t k = b; k < e; ++k) off.push_back(ci[k] - (int32_t)i);
            ptr.push_back((int64_t)off.size());
            ids.push_back(found);
        }
        pid[i] = found;
    }
    PD_TRY(dalloc(c, &c->gpat_id, (size_t)N));
    PD_TRY(dalloc(c, &c->gpat_ptr, ptr.size()));
    PD_TRY(dalloc(c, &c->gpat_off, std::max<size_t>(off.size(), 1)));
    PD_TRY(upload(c, c->gpat_id, pid.data(), sizeof(int32_t) * pid.size()));
    PD_TRY(upload(c, c->gpat_ptr, ptr.data(), sizeof(int64_t) * ptr.size()));
    if (!off.empty()) PD_TRY(upload(c, c->gpat_off, off.data(), sizeof(int32_t) * off.size()));
    c->have_gpat = true;
    gpat_apply(c);
    return PD_OK;
}

static void mls_release(pd_ctx* c) {
    for (void* p : {(void*)c->tptr, (void*)c->tj, (void*)c->tpos, (void*)c->cbptr, (void*)c->cbidx, (void*)c->coeff,
                    (void*)c->coeff32, (void*)c->csum})
        dfree(c, p);
    c->tptr = nullptr;
    c->tj = c->tpos = nullptr;
    c->cbptr = nullptr;
    c->cbidx = nullptr;
    c->coeff = nullptr;
    c->coeff32 = c->csum = nullptr;
    c->d.cbptr = nullptr;
    c->d.cbidx = nullptr;
    c->d.coeff = nullptr;
    c->d.coeff32 = c->d.csum = nullptr;
    c->have_mls = false;
    c->generation++;
}

// after new MLS data: the patterns and the SELL copy
static int mls_installed(pd_ctx* c) {
    c->d.cbptr = c->cbptr;
    c->d.cbidx = c->cbidx;
    c->d.coeff = c->coeff;
    c->d.coeff32 = c->coeff32;
    c->d.csum = c->csum;
    c->have_mls = true;
    c->generation++;
    PD_TRY(gpat_build(c));
    if (!c->have_gpat) c->gpat_opt = 0;  // the new lists do not repeat: plain lists
    gpat_apply(c);
    return sell_prepare(c);
}

// The lattice-stencil FP32 force: off (buffers freed, contiguous node blocks).
static void fsten_release(pd_ctx* c) {
    dfree(c, c->fst_u2);
    dfree(c, c->fst_mask);
    dfree(c, c->fst_tab);
    dfree(c, c->fst_box);
    dfree(c, c->fst_boxb);
    dfree(c, c->fst_wide);
    c->fst_wide = nullptr;
    c->d.sten_wide = nullptr;
    c->fst_box = nullptr;
    c->fst_boxb = nullptr;
    c->d.sten_box = nullptr;
    c->d.sten_boxb = nullptr;
    c->d.sten_nbox = 0;
    c->d.sten_ntiles = 0;
    c->fst_u2 = nullptr;
    c->fst_mask = nullptr;
    c->fst_tab = nullptr;
    c->fst_shape = 0;
    c->d.blk_cm = 0;
    c->d.sten_u2 = nullptr;
    c->d.sten_mask = nullptr;
    c->d.sten_tab = nullptr;
    c->d.sten_nu = c->d.sten_nw = 0;
    c->d.sten_np = 0;
    c->generation++;
}

// Builds the stencil S (every offset an unbroken family entry takes), the
// union list U2 = S u (S + e_x) of a node pair and the masks of every pair,
// checking on the device that the node ids follow x + nx (y + ny z) and that
// every family maps onto U2 in ascending order.
// The tiles of every box for the block shape (tw pairs x by 16 / tw rows x
// bz layers, tw = sten_tw of the box; runs of 128 pairs where sten_linear):
// first tile of each box into fst_box, their total into d.sten_ntiles.
static int fsten_tiles(pd_ctx* c, int by, int bz) {
    std::vector<int4> bx(c->box_dims.size());
    int64_t t = 0;
    for (size_t b = 0; b < bx.size(); ++b) {
        const int4 D = c->box_dims[b];
        const int npx = (D.x + 1) / 2, tw = pd::sten_tw(npx), byw = by * (16 / tw);
        bx[b] = make_int4(D.x, D.y, D.z, (int)t);
        if (pd::sten_linear(npx, D.y, D.z, tw, byw, bz))
            t += ((int64_t)npx * D.y * D.z + 127) / 128;
        else
            t += (int64_t)((npx + tw - 1) / tw) * ((D.y + byw - 1) / byw) * ((D.z + bz - 1) / bz);
        if (t > INT32_MAX) return fail(PD_ERR_ARG, "pd_set_option: too many stencil force tiles");
    }
    PD_TRY(upload(c, c->fst_box, bx.data(), sizeof(int4) * bx.size()));
    dfree(c, c->fst_wide);
    c->fst_wide = nullptr;
    c->d.sten_wide = nullptr;
    PD_TRY(dalloc(c, &c->fst_wide, (size_t)std::max<int64_t>(t, 1)));
    PD_CUDA_TRY(cudaMemsetAsync(c->fst_wide, 0, (size_t)std::max<int64_t>(t, 1), c->stream));
    c->d.sten_wide = c->fst_wide;
    c->d.sten_ntiles = t;
    return PD_OK;
}

static int fsten_prepare(pd_ctx* c, int shape) {
    static const int kBy[5] = {0, 8, 4, 2, 1};
    if (shape < 0 || shape > 4) return fail(PD_ERR_ARG, "pd_set_option: stencil force shape 0..4");
    if (shape == 0) {
        fsten_release(c);
        return PD_OK;
    }
    if (c->fst_mask) {  // built: only the block shape changes
        PD_TRY(fsten_tiles(c, kBy[shape], 8 / kBy[shape]));
        c->fst_shape = shape;
        c->d.sten_by = kBy[shape];
        c->d.sten_bz = 8 / kBy[shape];
        c->generation++;
        return PD_OK;
    }
    const int64_t NX = c->d.lat_nx, NY = c->d.lat_ny, NZ = c->d.lat_nz;
    const bool one_box = c->box_first.empty();
    if (c->d.cci || c->npt != 8 || !c->d.gc_host || !c->d.lat || !c->have_family || c->d.multimat || c->n == 0 ||
        (one_box && NX * NY * NZ != c->n))
        return fail(PD_ERR_ARG,
                    "pd_set_option: the stencil force needs 2x2x2 points, one material, a family and complete "
                    "box lattices");
    if (one_box) {
        c->box_dims.assign(1, make_int4((int)NX, (int)NY, (int)NZ, 0));
    }
    const std::vector<int64_t> firsts = one_box ? std::vector<int64_t>{0} : c->box_first;
    const int nbox = (int)c->box_dims.size();
    std::vector<longlong2> boxb(nbox);
    int64_t np = 0;
    for (int b = 0; b < nbox; ++b) {
        boxb[b] = make_longlong2(firsts[b], np);
        np += (int64_t)(c->box_dims[b].x + 1) / 2 * c->box_dims[b].y * c->box_dims[b].z;
    }
    {
        int rc0 = PD_OK;
        if ((rc0 = dalloc(c, &c->fst_box, nbox)) || (rc0 = dalloc(c, &c->fst_boxb, nbox)) ||
            (rc0 = upload(c, c->fst_boxb, boxb.data(), sizeof(longlong2) * nbox))) {
            fsten_release(c);
            return rc0;
        }
        c->d.sten_box = c->fst_box;
        c->d.sten_boxb = c->fst_boxb;
        c->d.sten_nbox = nbox;
        if ((rc0 = fsten_tiles(c, kBy[shape], 8 / kBy[shape])) != PD_OK) {
            fsten_release(c);
            return rc0;
        }
    }
    int* rad = reinterpret_cast<int*>(c->hscalar + 8);
    pd::launch_family_radius(c->d, reinterpret_cast<int*>(c->scal + pd::CG_NSLOT - 1), c->stream);
    if (cudaMemcpyAsync(rad, c->scal + pd::CG_NSLOT - 1, sizeof(int), cudaMemcpyDeviceToHost, c->stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(c->stream) != cudaSuccess) {
        fsten_release(c);
        return fail(PD_ERR_CUDA, "stencil force: family radius");
    }
    const int R = *rad;
    if (R > 16) {
        fsten_release(c);
        return fail(PD_ERR_ARG, "pd_set_option: family radius too large for the stencil force");
    }
    const int W = 2 * R + 1;
    int* dbits = nullptr;  // [W^3] bitmap, then the error word
    PD_TRY(dalloc(c, &dbits, (size_t)W * W * W + 1));
    int* derr = dbits + (size_t)W * W * W;
    auto done = [&](int rc) {
        dfree(c, dbits);
        if (rc != PD_OK) fsten_release(c);
        return rc;
    };
    if (cudaMemsetAsync(dbits, 0, sizeof(int) * ((size_t)W * W * W + 1), c->stream) != cudaSuccess)
        return done(fail(PD_ERR_CUDA, "stencil force: memset"));
    pd::launch_sten_offsets(c->d, R, dbits, derr, c->stream);
    std::vector<int> bits((size_t)W * W * W + 1);
    if (cudaMemcpyAsync(bits.data(), dbits, sizeof(int) * bits.size(), cudaMemcpyDeviceToHost, c->stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(c->stream) != cudaSuccess)
        return done(fail(PD_ERR_CUDA, "stencil force: offsets"));
    if (bits.back() != 0)
        return done(fail(PD_ERR_ARG, "pd_set_option: node ids do not follow the box lattice x + nx (y + ny z)"));
    // U2 in lin() order is ascending neighbour id for every node of every box:
    // two offsets that stay in a box of width nx differ by at most nx - 1 in
    // x, so their order by (oz, oy, ox) is their order by id in that box, and
    // lin() with the lattice's nx >= every box's nx keeps that order too.
    // S in ascending id offset, then U2 = S u (S + e_x)
    auto lin = [&](int ox, int oy, int oz) { return (int64_t)ox + NX * ((int64_t)oy + NY * oz); };
    std::vector<std::array<int, 3>> S;
    for (int oz = -R; oz <= R; ++oz)
        for (int oy = -R; oy <= R; ++oy)
            for (int ox = -R; ox <= R; ++ox)
                if (bits[(ox + R) + W * ((oy + R) + W * (oz + R))]) S.push_back({ox, oy, oz});
    auto by_lin = [&](const std::array<int, 3>& a, const std::array<int, 3>& b) {
        return lin(a[0], a[1], a[2]) < lin(b[0], b[1], b[2]);
    };
    std::sort(S.begin(), S.end(), by_lin);
    const int WX = W + 1;
    std::vector<int> sidx((size_t)WX * W * W, -1);  // offset from A over [-R, R+1] x [-R, R]^2 -> S index
    for (size_t k = 0; k < S.size(); ++k) sidx[(S[k][0] + R) + WX * ((S[k][1] + R) + W * (S[k][2] + R))] = (int)k;
    std::vector<std::array<int, 3>> U;
    for (int oz = -R; oz <= R; ++oz)
        for (int oy = -R; oy <= R; ++oy)
            for (int ox = -R; ox <= R + 1; ++ox) {
                const bool a = ox <= R && sidx[(ox + R) + WX * ((oy + R) + W * (oz + R))] >= 0;
                const bool b = ox - 1 >= -R && sidx[(ox - 1 + R) + WX * ((oy + R) + W * (oz + R))] >= 0;
                if (a || b) U.push_back({ox, oy, oz});
            }
    std::sort(U.begin(), U.end(), by_lin);
    if (U.size() > 512) return done(fail(PD_ERR_ARG, "pd_set_option: stencil of more than 512 pair offsets"));
    std::vector<int4> u2(U.size());
    std::vector<int> lut((size_t)WX * W * W, -1);
    for (size_t u = 0; u < U.size(); ++u) {
        const int ox = U[u][0], oy = U[u][1], oz = U[u][2];
        u2[u] = make_int4((int)lin(ox, oy, oz), ox, oy, oz);
        lut[(ox + R) + WX * ((oy + R) + W * (oz + R))] = (int)u;
    }
    const int nu = (int)U.size(), nw = (nu + 31) / 32;
    int* dlut = nullptr;
    int rc = PD_OK;
    if ((rc = dalloc(c, &c->fst_u2, std::max<size_t>(u2.size(), 1))) ||
        (rc = dalloc(c, &c->fst_mask, (size_t)2 * nw * np)) || (rc = dalloc(c, &dlut, lut.size())) ||
        (rc = dalloc(c, &c->fst_tab, (size_t)8 * nu)))
        return done(rc);
    auto done2 = [&](int r) {
        dfree(c, dlut);
        return done(r);
    };
    if ((rc = upload(c, c->fst_u2, u2.data(), sizeof(int4) * u2.size())) ||
        (rc = upload(c, dlut, lut.data(), sizeof(int) * lut.size())))
        return done2(rc);
    pd::Dev t = c->d;
    t.sten_u2 = c->fst_u2;
    t.sten_mask = c->fst_mask;
    t.sten_nu = nu;
    t.sten_nw = nw;
    t.sten_np = np;
    pd::launch_sten_masks(t, dlut, R, c->fst_mask, derr, c->stream);
    int err = 0;
    if (cudaMemcpyAsync(&err, derr, sizeof(int), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
        cudaStreamSynchronize(c->stream) != cudaSuccess)
        return done2(fail(PD_ERR_CUDA, "stencil force: masks"));
    if (err) return done2(fail(PD_ERR_ARG, "pd_set_option: a family does not map onto the lattice stencil"));
    t.sten_tab = c->fst_tab;
    if ((rc = pd::launch_sten_table(t, c->fst_tab, c->stream)) != PD_OK ||
        cudaStreamSynchronize(c->stream) != cudaSuccess)
        return done2(fail(PD_ERR_CUDA, "stencil force: geometry table"));
    t.blk_cm = 1;
    t.sten_by = kBy[shape];
    t.sten_bz = 8 / kBy[shape];
    c->d = t;
    c->fst_shape = shape;
    c->generation++;
    return done2(PD_OK);
}

static void install_family(pd_ctx* c, int64_t* frow, int32_t* fcol, uint8_t* fbr, int64_t* arow, int32_t* acol,
                           int64_t H, int64_t Ha) {
    dfree(c, c->frow); dfree(c, c->fcol); dfree(c, c->fbroken); dfree(c, c->arow); dfree(c, c->acol);
    c->frow = frow; c->fcol = fcol; c->fbroken = fbr; c->arow = arow; c->acol = acol;
    for (void* p : {(void*)frow, (void*)fcol, (void*)fbr, (void*)arow, (void*)acol}) c->owned.push_back(p);
    c->d.frow = frow; c->d.fcol = fcol; c->d.fbroken = fbr; c->d.arow = arow; c->d.acol = acol;
    c->H = H;
    c->Ha = Ha;
    c->have_family = true;
    c->have_ai = false;                            // its regions follow the family
    c->d.tile_x = c->d.tile_y = c->d.tile_z = 0;  // its family radius may have changed
    if (c->fst_mask) fsten_release(c);
    c->generation++;
}

// Node ranges offsets[b] .. offsets[b + 1] - 1 that each form a complete box
// lattice in id order (the specimens of a batch): the lattice-stencil force
// then runs on every box.  The dimensions come from the coordinates.
int pd_set_boxes(pd_ctx* c, int nbox, const int64_t* offsets) {
    if (!c) return fail(PD_ERR_ARG, "pd_set_boxes: null context");
    if (nbox < 0 || (nbox > 0 && !offsets)) return fail(PD_ERR_ARG, "pd_set_boxes: null offsets");
    std::vector<int64_t> first;
    std::vector<int4> dims;
    if (nbox > 0) {
        if (offsets[0] != 0 || offsets[nbox] != c->n)
            return fail(PD_ERR_ARG, "pd_set_boxes: the ranges must cover the nodes in order");
        std::vector<int32_t> lat;
        if (!lattice_positions(c->coords, c->n, c->d.dx, lat))
            return fail(PD_ERR_ARG, "pd_set_boxes: the nodes are not on one lattice");
        auto pos = [&](int64_t i, int* q) {
            q[0] = lat[i] & 2047;
            q[1] = (lat[i] >> 11) & 2047;
            q[2] = lat[i] >> 22;
        };
        for (int b = 0; b < nbox; ++b) {
            const int64_t f0 = offsets[b], f1 = offsets[b + 1];
            if (f1 <= f0) return fail(PD_ERR_ARG, "pd_set_boxes: empty or descending range");
            int o[3], q[3], ext[3] = {0, 0, 0};
            pos(f0, o);
            for (int64_t i = f0; i < f1; ++i) {
                pos(i, q);
                for (int a = 0; a < 3; ++a) {
                    if (q[a] < o[a]) return fail(PD_ERR_ARG, "pd_set_boxes: a range does not start at its corner");
                    ext[a] = std::max(ext[a], q[a] - o[a] + 1);
                }
            }
            if ((int64_t)ext[0] * ext[1] * ext[2] != f1 - f0)
                return fail(PD_ERR_ARG, "pd_set_boxes: a range is not a complete box");
            for (int64_t i = f0; i < f1; ++i) {
                pos(i, q);
                if (i != f0 + (q[0] - o[0]) + (int64_t)ext[0] * ((q[1] - o[1]) + (int64_t)ext[1] * (q[2] - o[2])))
                    return fail(PD_ERR_ARG, "pd_set_boxes: node ids do not follow x + nx (y + ny z) in a box");
            }
            first.push_back(f0);
            dims.push_back(make_int4(ext[0], ext[1], ext[2], 0));
        }
    }
    if (c->fst_mask) fsten_release(c);  // the next PD_OPT_FORCE_STENCIL builds on the boxes
    c->box_first = first;
    c->box_dims = dims;
    c->generation++;
    return PD_OK;
}

int pd_bond_search(pd_ctx* c, int64_t* num_halves, int64_t* num_broken, double* min_bond_length) {
    if (!c) return fail(PD_ERR_ARG, "pd_bond_search: null context");
    const int64_t N = c->n;
    pd::SearchGrid g{};
    double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    for (int a = 0; a < 3; ++a) { lo[a] = INFINITY; hi[a] = -INFINITY; }
    for (int64_t i = 0; i < N; ++i)
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], c->coords[3 * i + a]);
            hi[a] = std::max(hi[a], c->coords[3 * i + a]);
        }
    if (N == 0)
        for (int a = 0; a < 3; ++a) lo[a] = hi[a] = 0.0;
    g.h = c->d.delta + c->d.dx;  // >= horizon + tolerance + half cell diagonal
    int64_t ncell = 1;
    for (int a = 0; a < 3; ++a) {
        g.lo[a] = lo[a];
        g.nc[a] = (int64_t)std::floor((hi[a] - lo[a]) / g.h) + 1;
        ncell *= g.nc[a];
    }
    // Morton rank of every cell
    std::vector<std::pair<uint64_t, int64_t>> keys(ncell);
    for (int64_t z = 0; z < g.nc[2]; ++z)
        for (int64_t y = 0; y < g.nc[1]; ++y)
            for (int64_t xx = 0; xx < g.nc[0]; ++xx) {
                int64_t lin = (z * g.nc[1] + y) * g.nc[0] + xx;
                keys[lin] = {morton3(xx, y, z), lin};
            }
    std::sort(keys.begin(), keys.end());
    std::vector<int32_t> rank(ncell);
    for (int64_t r = 0; r < ncell; ++r) rank[keys[r].second] = (int32_t)r;
    int32_t* drank = nullptr;
    PD_TRY(dalloc(c, &drank, ncell));
    int rc = upload(c, drank, rank.data(), sizeof(int32_t) * ncell);
    if (rc != PD_OK) { dfree(c, drank); return rc; }
    double* sl = c->dslits;
    int64_t *frow, *arow;
    int32_t *fcol, *acol;
    uint8_t* fbr;
    int64_t nh = 0, nb = 0;
    double mb = 0.0;
    rc = pd::bond_search(c->d, g, drank, ncell, c->nslit, sl, &frow, &fcol, &fbr, &arow, &acol, &nh, &nb, &mb,
                         c->stream);
    dfree(c, drank);
    if (rc != PD_OK) return rc;
    install_family(c, frow, fcol, fbr, arow, acol, nh, nh - nb);
    if (num_halves) *num_halves = nh;
    if (num_broken) *num_broken = nb;
    if (min_bond_length) *min_bond_length = mb;
    return PD_OK;
}

int pd_get_family(pd_ctx* c, int64_t* row_ptr, int32_t* col, uint8_t* broken) {
    if (!c || !c->have_family) return fail(PD_ERR_ARG, "pd_get_family: no family");
    if (row_ptr) PD_CUDA_TRY(cudaMemcpyAsync(row_ptr, c->frow, sizeof(int64_t) * (c->n + 1), cudaMemcpyDeviceToHost, c->stream));
    if (col) PD_CUDA_TRY(cudaMemcpyAsync(col, c->fcol, sizeof(int32_t) * c->H, cudaMemcpyDeviceToHost, c->stream));
    if (broken) PD_CUDA_TRY(cudaMemcpyAsync(broken, c->fbroken, c->H, cudaMemcpyDeviceToHost, c->stream));
    PD_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return PD_OK;
}

int pd_set_family(pd_ctx* c, const int64_t* row_ptr, const int32_t* col, const uint8_t* broken) {
    if (!c || !row_ptr || (!col && row_ptr[c->n] > 0)) return fail(PD_ERR_ARG, "pd_set_family: null argument");
    const int64_t N = c->n, H = row_ptr[N];
    if (row_ptr[0] != 0 || H < 0) return fail(PD_ERR_ARG, "pd_set_family: bad row_ptr");
    for (int64_t i = 0; i < N; ++i)
        if (row_ptr[i + 1] < row_ptr[i]) return fail(PD_ERR_ARG, "pd_set_family: row_ptr not monotone");
    for (int64_t p = 0; p < H; ++p)
        if (col[p] < 0 || col[p] >= N) return fail(PD_ERR_ARG, "pd_set_family: column out of range");
    std::vector<int64_t> ar(N + 1, 0);
    std::vector<int32_t> ac;
    std::vector<uint8_t> br(std::max<int64_t>(H, 1), 0);
    if (broken) std::copy(broken, broken + H, br.begin());
    ac.reserve(H);
    for (int64_t i = 0; i < N; ++i) {
        for (int64_t p = row_ptr[i]; p < row_ptr[i + 1]; ++p)
            if (!br[p]) ac.push_back(col[p]);
        ar[i + 1] = (int64_t)ac.size();
    }
    int64_t *frow, *arow;
    int32_t *fcol, *acol;
    uint8_t* fbr;
    PD_TRY(dalloc(c, &frow, N + 1));
    PD_TRY(dalloc(c, &fcol, H));
    PD_TRY(dalloc(c, &fbr, H));
    PD_TRY(dalloc(c, &arow, N + 1));
    PD_TRY(dalloc(c, &acol, ac.size()));
    for (void* p : {(void*)frow, (void*)fcol, (void*)fbr, (void*)arow, (void*)acol}) {
        auto it = std::find(c->owned.begin(), c->owned.end(), p);
        c->owned.erase(it);
    }
    PD_TRY(upload(c, frow, row_ptr, sizeof(int64_t) * (N + 1)));
    if (H) PD_TRY(upload(c, fcol, col, sizeof(int32_t) * H));
    if (H) PD_TRY(upload(c, fbr, br.data(), H));
    PD_TRY(upload(c, arow, ar.data(), sizeof(int64_t) * (N + 1)));
    if (!ac.empty()) PD_TRY(upload(c, acol, ac.data(), sizeof(int32_t) * ac.size()));
    install_family(c, frow, fcol, fbr, arow, acol, H, (int64_t)ac.size());
    return PD_OK;
}

int pd_set_bdry_eff(pd_ctx* c, const double* bE) {
    if (!c || !bE) return fail(PD_ERR_ARG, "pd_set_bdry_eff: null argument");
    PD_TRY(upload(c, (void*)c->d.bdry, bE, sizeof(double) * c->n));
    c->bdry_host.assign(bE, bE + c->n);
    c->d.bdry_on = 0;
    for (int64_t i = 0; i < c->n; ++i) c->d.bdry_on |= (bE[i] != 1.0);
    c->generation++;
    return upload_static_f32(c);
}

int pd_set_mls(pd_ctx* c, const int64_t* cb_ptr, const int32_t* cb_idx, const double* coeff) {
    if (!c || !cb_ptr || !cb_idx || !coeff) return fail(PD_ERR_ARG, "pd_set_mls: null argument");
    if (!c->d.mls) return fail(PD_ERR_ARG, "pd_set_mls: MLS is off for this integration scheme");
    const int64_t N = c->n, T = cb_ptr[N];
    const int npt = c->npt;
    if (cb_ptr[0] != 0) return fail(PD_ERR_ARG, "pd_set_mls: bad cb_ptr");
    for (int64_t i = 0; i < N; ++i)
        if (cb_ptr[i + 1] < cb_ptr[i]) return fail(PD_ERR_ARG, "pd_set_mls: cb_ptr not monotone");
    for (int64_t k = 0; k < T; ++k)
        if (cb_idx[k] < 0 || cb_idx[k] >= N) return fail(PD_ERR_ARG, "pd_set_mls: contributor out of range");
    // re-layout [node][point][contributor] -> [node][contributor][point]
    std::vector<double> co((size_t)T * npt);
    std::vector<float> co32((size_t)T * npt), cs((size_t)N * npt);
    for (int64_t i = 0; i < N; ++i) {
        const int64_t b = cb_ptr[i], nc = cb_ptr[i + 1] - b;
        for (int g = 0; g < npt; ++g) {
            double s = 0.0;
            for (int64_t k = 0; k < nc; ++k) {
                const double v = coeff[b * npt + (int64_t)g * nc + k];
                co[(b + k) * npt + g] = v;
                co32[(b + k) * npt + g] = (float)v;
                s += v;
            }
            cs[i * npt + g] = (float)(s - 1.0);
        }
    }
    c->cbptr_host.assign(cb_ptr, cb_ptr + N + 1);
    c->cbidx_host.assign(cb_idx, cb_idx + T);
    mls_release(c);
    PD_TRY(dalloc(c, &c->cbptr, N + 1));
    PD_TRY(dalloc(c, &c->cbidx, T));
    PD_TRY(dalloc(c, &c->coeff, (size_t)T * npt));
    PD_TRY(dalloc(c, &c->coeff32, (size_t)T * npt));
    PD_TRY(dalloc(c, &c->csum, (size_t)N * npt));
    PD_TRY(upload(c, c->cbptr, cb_ptr, sizeof(int64_t) * (N + 1)));
    if (T) PD_TRY(upload(c, c->cbidx, cb_idx, sizeof(int32_t) * T));
    if (T) PD_TRY(upload(c, c->coeff, co.data(), sizeof(double) * co.size()));
    if (T) PD_TRY(upload(c, c->coeff32, co32.data(), sizeof(float) * co32.size()));
    PD_TRY(upload(c, c->csum, cs.data(), sizeof(float) * cs.size()));
    return mls_installed(c);
}

// The MLS data of InitIntegrationPoint computed on the device (k_mls_contrib,
// k_mls_coeff) from the context's family and coordinates, or from the given
// MLS coordinates (a batch: every specimen in its own frame).
int pd_mls_setup(pd_ctx* c, double rw, const double* mls_coords, int64_t* num_contrib) {
    if (!c) return fail(PD_ERR_ARG, "pd_mls_setup: null context");
    if (!c->d.mls || c->d.cci) return fail(PD_ERR_ARG, "pd_mls_setup: MLS is off for this integration scheme");
    if (!c->have_family) return fail(PD_ERR_ARG, "pd_mls_setup: no family (pd_bond_search or pd_set_family first)");
    if (!(rw > 0.0) || c->abscis.empty()) return fail(PD_ERR_ARG, "pd_mls_setup: support size or Gauss rule");
    const int64_t N = c->n;
    const int n1 = (int)c->abscis.size();
    mls_release(c);
    double *xm = nullptr, *dab = nullptr;
    int64_t* cnt = nullptr;
    auto cleanup = [&]() { dfree(c, xm); dfree(c, dab); dfree(c, cnt); };
    int rc = PD_OK;
    if ((rc = dalloc(c, &cnt, (size_t)std::max<int64_t>(N, 1))) || (rc = dalloc(c, &dab, (size_t)n1)) ||
        (rc = dalloc(c, &c->cbptr, (size_t)N + 1)) || (rc = upload(c, dab, c->abscis.data(), sizeof(double) * n1))) {
        cleanup();
        return rc;
    }
    const double* xsrc = c->d.x;
    if (mls_coords) {
        if ((rc = dalloc(c, &xm, (size_t)(3 * N))) || (rc = upload_vec3(c, xm, mls_coords))) {
            cleanup();
            return rc;
        }
        xsrc = xm;
    }
    struct Alloc {
        static void* fn(void* ctx, size_t bytes) {
            char* p = nullptr;
            return dalloc(static_cast<pd_ctx*>(ctx), &p, bytes) == PD_OK ? (void*)p : nullptr;
        }
    };
    int64_t T = 0, bad = -1;
    rc = pd::mls_setup(c->d, xsrc, rw, dab, n1, cnt, c->cbptr, &c->cbidx, &c->coeff, &c->coeff32, &c->csum, &T, &bad,
                       &Alloc::fn, c, c->stream);
    cleanup();
    if (rc == PD_ERR_SINGULAR) {
        mls_release(c);
        const std::string msg =
            "pdMatrix::Gauss: Singular Matrix (MLS moment matrix of node " + std::to_string(bad) + ")";
        return fail(PD_ERR_SINGULAR, msg.c_str());
    }
    if (rc != PD_OK) {
        mls_release(c);
        return fail(rc, "pd_mls_setup: device setup failed");
    }
    c->cbptr_host.resize((size_t)N + 1);
    c->cbidx_host.resize((size_t)T);
    PD_CUDA_TRY(cudaMemcpy(c->cbptr_host.data(), c->cbptr, sizeof(int64_t) * (N + 1), cudaMemcpyDeviceToHost));
    if (T) PD_CUDA_TRY(cudaMemcpy(c->cbidx_host.data(), c->cbidx, sizeof(int32_t) * T, cudaMemcpyDeviceToHost));
    if (num_contrib) *num_contrib = T;
    return mls_installed(c);
}

// Half-space bond-force sums of PostAFD (k_afd_gauss, k_afd_items).
int pd_afd(pd_ctx* c, const double* U, const double* bdry_eff, int64_t n_items, const int64_t* item_i,
           const int64_t* item_s, const int32_t* item_dir, double* force) {
    if (!c || !U || !bdry_eff || n_items < 0 || (n_items > 0 && (!item_i || !item_s || !item_dir || !force)))
        return fail(PD_ERR_ARG, "pd_afd: null argument");
    if (!c->have_family) return fail(PD_ERR_ARG, "pd_afd: no family");
    if (!c->d.cci && c->d.mls && !c->have_mls) return fail(PD_ERR_ARG, "pd_afd: no MLS data");
    if (!c->d.cci && (c->abscis.empty() || c->gweights.size() != c->abscis.size()))
        return fail(PD_ERR_ARG, "pd_afd: no Gauss rule");
    const int64_t N = c->n;
    for (int64_t k = 0; k < n_items; ++k)
        if (item_i[k] < 0 || item_i[k] >= N || item_s[k] < 0 || item_s[k] >= N || item_dir[k] < 1 || item_dir[k] > 3)
            return fail(PD_ERR_ARG, "pd_afd: item out of range");
    if (n_items == 0 || N == 0) return PD_OK;
    const int n1 = c->d.cci ? 1 : (int)c->abscis.size();
    double *Ud = nullptr, *bEd = nullptr, *ug = nullptr, *ab = nullptr, *wt = nullptr, *out = nullptr;
    int64_t *ii = nullptr, *ss = nullptr;
    int32_t* dd = nullptr;
    auto cleanup = [&]() {
        for (void* p : {(void*)Ud, (void*)bEd, (void*)ug, (void*)ab, (void*)wt, (void*)out, (void*)ii, (void*)ss,
                        (void*)dd})
            dfree(c, p);
    };
    const std::vector<double> one{0.0};
    const std::vector<double> two{2.0};
    const std::vector<double>& av = c->d.cci ? one : c->abscis;
    const std::vector<double>& wv = c->d.cci ? two : c->gweights;
    int rc = PD_OK;
    if ((rc = dalloc(c, &Ud, (size_t)(3 * N))) || (rc = dalloc(c, &bEd, (size_t)N)) ||
        (rc = dalloc(c, &ug, (size_t)(3 * N * c->npt))) || (rc = dalloc(c, &ab, (size_t)n1)) ||
        (rc = dalloc(c, &wt, (size_t)n1)) || (rc = dalloc(c, &out, (size_t)(3 * n_items))) ||
        (rc = dalloc(c, &ii, (size_t)n_items)) || (rc = dalloc(c, &ss, (size_t)n_items)) ||
        (rc = dalloc(c, &dd, (size_t)n_items)) || (rc = upload_vec3(c, Ud, U)) ||
        (rc = upload(c, bEd, bdry_eff, sizeof(double) * N)) || (rc = upload(c, ab, av.data(), sizeof(double) * n1)) ||
        (rc = upload(c, wt, wv.data(), sizeof(double) * n1)) ||
        (rc = upload(c, ii, item_i, sizeof(int64_t) * n_items)) ||
        (rc = upload(c, ss, item_s, sizeof(int64_t) * n_items)) ||
        (rc = upload(c, dd, item_dir, sizeof(int32_t) * n_items))) {
        cleanup();
        return rc;
    }
    rc = pd::afd_forces(c->d, Ud, bEd, ug, ab, wt, n1, n_items, ii, ss, dd, out, c->stream);
    if (rc == PD_OK) {
        const cudaError_t e = cudaMemcpyAsync(force, out, sizeof(double) * 3 * n_items, cudaMemcpyDeviceToHost,
                                              c->stream);
        if (e != cudaSuccess || cudaStreamSynchronize(c->stream) != cudaSuccess) rc = PD_ERR_CUDA;
    }
    cleanup();
    return rc == PD_OK ? PD_OK : fail(rc, "pd_afd: device computation failed");
}

// Adaptive-trapezoid data: the regions of every full-family entry, the MLS
// contributors and tables (or, without MLS, the check that every family node
// carries a displacement gradient), and the per-entry work buffers.
int pd_set_ai(pd_ctx* c, int mls, const int64_t* reg_ptr, const pd_ai_region* regions, const int64_t* cb_ptr,
              const int32_t* cb_idx, const int64_t* tab_ptr, const double* tab_coeff) {
    if (!c || !reg_ptr) return fail(PD_ERR_ARG, "pd_set_ai: null argument");
    if (!c->d.ai) return fail(PD_ERR_ARG, "pd_set_ai: the context was not created with PD_INTG_AI");
    if (!c->have_family) return fail(PD_ERR_ARG, "pd_set_ai: no family (pd_bond_search or pd_set_family first)");
    const int64_t N = c->n, H = c->H;
    if (reg_ptr[0] != 0) return fail(PD_ERR_ARG, "pd_set_ai: bad reg_ptr");
    for (int64_t p = 0; p < H; ++p)
        if (reg_ptr[p + 1] < reg_ptr[p]) return fail(PD_ERR_ARG, "pd_set_ai: reg_ptr not monotone");
    const int64_t R = reg_ptr[H];
    if (R > 0 && !regions) return fail(PD_ERR_ARG, "pd_set_ai: null regions");
    for (int64_t r = 0; r < R; ++r) {
        const pd_ai_region& g = regions[r];
        const int a0 = g.axis[0], a1 = g.axis[1], a2 = g.axis[2];
        bool ok = a0 < 3 && a1 < 3 && a2 < 3 && a0 != a1 && a0 != a2 && a1 != a2;
        for (int k = 0; k < 2; ++k) ok = ok && (g.lim[k] < 6 || (g.lim[k] >= 8 && g.lim[k] < 44));
        for (int k = 2; k < 4; ++k) ok = ok && (g.lim[k] < 6 || (g.lim[k] >= 8 && g.lim[k] < 14));
        if (!ok) return fail(PD_ERR_ARG, "pd_set_ai: bad region axes or limit codes");
    }
    std::vector<int64_t> frow(N + 1);
    std::vector<int32_t> fcol(std::max<int64_t>(H, 1));
    std::vector<uint8_t> fbr(std::max<int64_t>(H, 1));
    PD_TRY(pd_get_family(c, frow.data(), fcol.data(), fbr.data()));
    // trapezoid points of every entry: the energy slots, and the work of
    // one force stage (the unbroken entries)
    int64_t points = 0;
    std::vector<int64_t> eptr(H + 1, 0);
    {
        struct Count {
            void operator()(const double*, int, double* f) const { f[0] = f[1] = f[2] = 0.0; }
        } none;
        for (int64_t i = 0; i < N; ++i)
            for (int64_t p = frow[i]; p < frow[i + 1]; ++p) {
                const int64_t j = fcol[p];
                double xj[3], f[3];
                int64_t np = 0;
                for (int a = 0; a < 3; ++a) xj[a] = c->coords[3 * j + a] - c->coords[3 * i + a];
                for (int64_t r = reg_ptr[p]; r < reg_ptr[p + 1]; ++r)
                    np += pd_ai::region(regions[r], c->d.ai_n, xj, c->d.delta, c->d.dx, none, f);
                eptr[p + 1] = eptr[p] + np;
                if (!fbr[p]) points += np;
            }
    }
    // work order of the bond kernel: entries grouped by region count and
    // points, so the threads of a warp walk the same loop structure
    std::vector<int32_t> order(std::max<int64_t>(H, 1));
    for (int64_t p = 0; p < H; ++p) order[p] = (int32_t)p;
    std::stable_sort(order.begin(), order.begin() + H, [&](int32_t a, int32_t b) {
        const int64_t ra = reg_ptr[a + 1] - reg_ptr[a], rb = reg_ptr[b + 1] - reg_ptr[b];
        if (ra != rb) return ra > rb;
        return (eptr[a + 1] - eptr[a]) > (eptr[b + 1] - eptr[b]);
    });
    std::vector<int32_t> row(std::max<int64_t>(H, 1));
    std::vector<int64_t> mirror(std::max<int64_t>(H, 1));
    for (int64_t i = 0; i < N; ++i)
        for (int64_t p = frow[i]; p < frow[i + 1]; ++p) {
            row[p] = (int32_t)i;
            const int64_t j = fcol[p];
            const int32_t* b = fcol.data() + frow[j];
            const int32_t* e = fcol.data() + frow[j + 1];
            const int32_t* q = std::lower_bound(b, e, (int32_t)i);
            if (q == e || *q != i) return fail(PD_ERR_ARG, "pd_set_ai: the family is not symmetric");
            mirror[p] = q - fcol.data();
        }
    int64_t T = 0, ncoef = 0;
    std::vector<int32_t> tnode;
    std::vector<int64_t> coff(N + 1, 0);
    if (mls) {
        if (!cb_ptr || !cb_idx || !tab_ptr || !tab_coeff) return fail(PD_ERR_ARG, "pd_set_ai: null MLS data");
        if (cb_ptr[0] != 0 || tab_ptr[0] != 0) return fail(PD_ERR_ARG, "pd_set_ai: bad cb_ptr / tab_ptr");
        for (int64_t i = 0; i < N; ++i) {
            if (cb_ptr[i + 1] < cb_ptr[i] || tab_ptr[i + 1] < tab_ptr[i])
                return fail(PD_ERR_ARG, "pd_set_ai: cb_ptr / tab_ptr not monotone");
            coff[i + 1] = coff[i] + (tab_ptr[i + 1] - tab_ptr[i]) * (cb_ptr[i + 1] - cb_ptr[i]);
        }
        for (int64_t k = 0; k < cb_ptr[N]; ++k)
            if (cb_idx[k] < 0 || cb_idx[k] >= N) return fail(PD_ERR_ARG, "pd_set_ai: contributor out of range");
        T = tab_ptr[N];
        ncoef = coff[N];
        tnode.resize(std::max<int64_t>(T, 1));
        for (int64_t i = 0; i < N; ++i)
            for (int64_t e = tab_ptr[i]; e < tab_ptr[i + 1]; ++e) tnode[e] = (int32_t)i;
    } else {
        for (int64_t p = 0; p < H; ++p) {
            const int b = c->bc_host[fcol[p]];
            if (b < 0 || c->bctype_host[b] != PD_BC_DISPLGRAD)
                return fail(PD_ERR_ARG, "pd_set_ai: without MLS every family node needs a displacement-gradient "
                                        "condition (pdIntgManager2.cpp:211-235)");
        }
    }
    for (void* q : c->ai_bufs) dfree(c, q);
    c->ai_bufs.clear();
    c->have_ai = false;
    pd::Dev& d = c->d;
    int64_t *rptr = nullptr, *mir = nullptr, *tptr = nullptr, *cof = nullptr, *cbp = nullptr;
    int32_t *rw = nullptr, *tn = nullptr, *cbi = nullptr, *fl = nullptr, *dmg = nullptr;
    pd_ai_region* reg = nullptr;
    double *tco = nullptr, *au = nullptr, *F = nullptr, *ae = nullptr;
    int64_t* ep = nullptr;
    uint8_t* brk = nullptr;
    int* err = nullptr;
    auto track = [&](void* q) { c->ai_bufs.push_back(q); };
    PD_TRY(dalloc(c, &rptr, H + 1)); track(rptr);
    PD_TRY(dalloc(c, &reg, R)); track(reg);
    PD_TRY(dalloc(c, &rw, H)); track(rw);
    PD_TRY(dalloc(c, &mir, H)); track(mir);
    PD_TRY(dalloc(c, &F, 3 * H)); track(F);
    PD_TRY(dalloc(c, &fl, H)); track(fl);
    PD_TRY(dalloc(c, &brk, H)); track(brk);
    PD_TRY(dalloc(c, &dmg, N)); track(dmg);
    PD_TRY(dalloc(c, &err, 1)); track(err);
    PD_TRY(dalloc(c, &ep, H + 1)); track(ep);
    int32_t* ord = nullptr;
    PD_TRY(dalloc(c, &ord, H)); track(ord);
    if (H) PD_TRY(upload(c, ord, order.data(), sizeof(int32_t) * H));
    PD_TRY(dalloc(c, &ae, eptr[H])); track(ae);
    PD_TRY(upload(c, ep, eptr.data(), sizeof(int64_t) * (H + 1)));
    PD_TRY(upload(c, rptr, reg_ptr, sizeof(int64_t) * (H + 1)));
    if (R) PD_TRY(upload(c, reg, regions, sizeof(pd_ai_region) * R));
    if (H) {
        PD_TRY(upload(c, rw, row.data(), sizeof(int32_t) * H));
        PD_TRY(upload(c, mir, mirror.data(), sizeof(int64_t) * H));
        PD_CUDA_TRY(cudaMemcpyAsync(brk, c->fbroken, H, cudaMemcpyDeviceToDevice, c->stream));
    }
    PD_CUDA_TRY(cudaMemsetAsync(dmg, 0, sizeof(int32_t) * N, c->stream));
    PD_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(int), c->stream));
    if (mls) {
        PD_TRY(dalloc(c, &cbp, N + 1)); track(cbp);
        PD_TRY(dalloc(c, &cbi, cb_ptr[N])); track(cbi);
        PD_TRY(dalloc(c, &tptr, N + 1)); track(tptr);
        PD_TRY(dalloc(c, &cof, N + 1)); track(cof);
        PD_TRY(dalloc(c, &tn, T)); track(tn);
        PD_TRY(dalloc(c, &tco, ncoef)); track(tco);
        PD_TRY(dalloc(c, &au, 3 * T)); track(au);
        PD_TRY(upload(c, cbp, cb_ptr, sizeof(int64_t) * (N + 1)));
        if (cb_ptr[N]) PD_TRY(upload(c, cbi, cb_idx, sizeof(int32_t) * cb_ptr[N]));
        PD_TRY(upload(c, tptr, tab_ptr, sizeof(int64_t) * (N + 1)));
        PD_TRY(upload(c, cof, coff.data(), sizeof(int64_t) * (N + 1)));
        if (T) PD_TRY(upload(c, tn, tnode.data(), sizeof(int32_t) * T));
        if (ncoef) PD_TRY(upload(c, tco, tab_coeff, sizeof(double) * ncoef));
        PD_CUDA_TRY(cudaMemsetAsync(au, 0, sizeof(double) * 3 * std::max<int64_t>(T, 1), c->stream));
        c->cbptr_host.assign(cb_ptr, cb_ptr + N + 1);
        c->cbidx_host.assign(cb_idx, cb_idx + cb_ptr[N]);
    }
    PD_CUDA_TRY(cudaStreamSynchronize(c->stream));
    d.ai_mls = mls ? 1 : 0;
    d.ai_nent = H;
    d.ai_ntab = T;
    d.ai_rptr = rptr;
    d.ai_reg = reg;
    d.ai_row = rw;
    d.ai_mirror = mir;
    d.ai_F = F;
    d.ai_fail = fl;
    d.ai_brk = brk;
    d.ai_dmg = dmg;
    d.ai_err = err;
    d.ai_eptr = ep;
    d.ai_order = ord;
    d.ai_e = ae;
    d.ai_tptr = tptr;
    d.ai_coff = cof;
    d.ai_tnode = tn;
    d.ai_tcoef = tco;
    d.ai_u = au;
    d.cbptr = cbp;
    d.cbidx = cbi;
    c->have_ai = true;
    c->ai_points = points;
    c->generation++;
    return PD_OK;
}

int pd_get_damage(pd_ctx* c, uint8_t* broken, int32_t* count) {
    if (!c) return fail(PD_ERR_ARG, "pd_get_damage: null context");
    const bool ai = c->d.ai && c->have_ai;
    if (broken) {
        if (!c->have_family) return fail(PD_ERR_ARG, "pd_get_damage: no family");
        if (c->H)
            PD_CUDA_TRY(cudaMemcpyAsync(broken, ai ? c->d.ai_brk : c->fbroken, c->H, cudaMemcpyDeviceToHost,
                                        c->stream));
    }
    if (count) {
        if (ai) PD_CUDA_TRY(cudaMemcpyAsync(count, c->d.ai_dmg, sizeof(int32_t) * c->n, cudaMemcpyDeviceToHost,
                                            c->stream));
        else std::fill(count, count + c->n, 0);
    }
    PD_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return PD_OK;
}

// The MLS data out, in the layout pd_set_mls takes (coeff [node][point][contributor]).
int pd_get_mls(pd_ctx* c, int64_t* cb_ptr, int32_t* cb_idx, double* coeff) {
    if (!c || !cb_ptr) return fail(PD_ERR_ARG, "pd_get_mls: null argument");
    if (!c->have_mls) return fail(PD_ERR_ARG, "pd_get_mls: no MLS data");
    const int64_t N = c->n, T = c->cbptr_host.empty() ? 0 : c->cbptr_host[N];
    const int npt = c->npt;
    std::memcpy(cb_ptr, c->cbptr_host.data(), sizeof(int64_t) * (N + 1));
    if (cb_idx && T) std::memcpy(cb_idx, c->cbidx_host.data(), sizeof(int32_t) * T);
    if (coeff && T) {
        std::vector<double> co((size_t)T * npt);
        PD_CUDA_TRY(cudaMemcpy(co.data(), c->coeff, sizeof(double) * co.size(), cudaMemcpyDeviceToHost));
        for (int64_t i = 0; i < N; ++i) {
            const int64_t b = c->cbptr_host[i], nc = c->cbptr_host[i + 1] - b;
            for (int64_t k = 0; k < nc; ++k)
                for (int g = 0; g < npt; ++g) coeff[b * npt + (int64_t)g * nc + k] = co[(b + k) * npt + g];
        }
    }
    return PD_OK;
}

int pd_mls_size(pd_ctx* c, int64_t* num_contrib) {
    if (!c || !num_contrib) return fail(PD_ERR_ARG, "pd_mls_size: null argument");
    *num_contrib = c->have_mls && !c->cbptr_host.empty() ? c->cbptr_host[c->n] : 0;
    return PD_OK;
}

int pd_set_precision(pd_ctx* c, int p) {
    if (!c || (p != PD_PREC_FP64 && p != PD_PREC_FP32C && p != PD_PREC_FP64A))
        return fail(PD_ERR_ARG, "pd_set_precision: bad argument");
    if (c->d.ai && p != PD_PREC_FP64)
        return fail(PD_ERR_ARG, "pd_set_precision: the AI form runs the FP64 drop-in arithmetic only");
    c->precision = p;
    c->d.acc_stretch = p == PD_PREC_FP64A;
    return PD_OK;
}

int pd_set_option(pd_ctx* c, int option, int64_t value) {
    if (!c) return fail(PD_ERR_ARG, "pd_set_option: null context");
    if (value < 0) return fail(PD_ERR_ARG, "pd_set_option: negative value");
    switch (option) {
        case PD_OPT_F64_LANES_BELOW: c->d.f64_lanes_below = value; break;
        case PD_OPT_TILE: {
            const int bx = (int)(value & 0xff), by = (int)((value >> 8) & 0xff), bz = (int)((value >> 16) & 0xff);
            if (bx < 1 || bx > 6 || by > 6 || bz > 6) return fail(PD_ERR_ARG, "pd_set_option: tile exponents");
            std::vector<int32_t> ord = tiled_order(c->coords, c->n, c->d.dx, bx, by, bz);
            PD_TRY(upload(c, (void*)c->d.order, ord.data(), sizeof(int32_t) * c->n));
            PD_CUDA_TRY(cudaStreamSynchronize(c->stream));
            c->tile = value;
            if (c->d.sell_on) PD_TRY(sell_prepare(c));
            break;
        }
        case PD_OPT_PERSIST_BLOCKS_PER_SM:
            if (value > 32) return fail(PD_ERR_ARG, "pd_set_option: blocks per SM");
            c->persist_per_sm = (int)value;
            break;
        case PD_OPT_STATIC_STENCIL:
            if (value > 1) return fail(PD_ERR_ARG, "pd_set_option: 0 or 1");
            c->static_stencil_opt = (int)value;
            break;
        case PD_OPT_ADJOINT_VJP32:
            if (value > 1) return fail(PD_ERR_ARG, "pd_set_option: 0 or 1");
            c->adj_vjp32 = (int)value;
            return PD_OK;
        case PD_OPT_STATIC_F32_BELOW:
            if (value > 1000000000) return fail(PD_ERR_ARG, "pd_set_option: 0..1e9");
            c->static_f32_below = value;
            return PD_OK;
        case PD_OPT_STATIC_SPLIT:
            if (value != 0 && value != 2 && value != 4 && value != 8)
                return fail(PD_ERR_ARG, "pd_set_option: 0, 2, 4 or 8");
            c->static_split = (int)value;
            c->sten.ndr = c->sten.ndcol > 0 ? (int)value : 0;
            return PD_OK;
        case PD_OPT_GATHER_PER_POINT:
            if (value > 1) return fail(PD_ERR_ARG, "pd_set_option: 0 or 1");
            c->d.gather_per_point = (int)value;
            break;
        case PD_OPT_PERSIST_WAIT_US:
            if (value < 1000 || value > 60000000) return fail(PD_ERR_ARG, "pd_set_option: wait 1e3..6e7 us");
            c->persist_wait_us = value;
            break;
        case PD_OPT_PERSIST_TEST_STALL:
            if (value > 1) return fail(PD_ERR_ARG, "pd_set_option: 0 or 1");
            c->persist_stall = (int)value;
            break;
        case PD_OPT_FORCE_QUAD:
            if (value > 1) return fail(PD_ERR_ARG, "pd_set_option: 0 or 1");
            c->d.force_quad = (int)value;
            break;
        case PD_OPT_GATHER_STENCIL:
            if (value > 1) return fail(PD_ERR_ARG, "pd_set_option: 0 or 1");
            if (value && !c->have_gpat)
                return fail(PD_ERR_ARG, "pd_set_option: the MLS contributor lists do not repeat (no patterns)");
            c->gpat_opt = (int)value;
            gpat_apply(c);
            break;
        case PD_OPT_STATIC_PRECOND:  // the static options leave the prepared stencil valid
            if (value > 1) return fail(PD_ERR_ARG, "pd_set_option: 0 or 1");
            c->static_precond = (int)value;
            return PD_OK;
        case PD_OPT_FORCE_STENCIL:
            if (value > 4) return fail(PD_ERR_ARG, "pd_set_option: stencil force shape 0..4");
            PD_TRY(fsten_prepare(c, (int)value));
            break;
        case PD_OPT_GATHER_SELL:
            if (value > 1) return fail(PD_ERR_ARG, "pd_set_option: 0 or 1");
            if ((int)value != c->d.sell_on) {
                c->d.sell_on = (int)value;
                PD_TRY(sell_prepare(c));
            }
            break;
        case PD_OPT_FORCE_TILE: {
            if (value == 0) {
                c->d.tile_x = c->d.tile_y = c->d.tile_z = 0;
                break;
            }
            const int tx = (int)(value & 0xff), ty = (int)((value >> 8) & 0xff), tz = (int)((value >> 16) & 0xff);
            const int threads = tx / 2 * ty * tz;
            if (tx < 2 || tx % 2 || ty < 1 || tz < 1 || threads < 32 || threads > 256)
                return fail(PD_ERR_ARG, "pd_set_option: tile (x even, 32..256 node pairs)");
            if (c->d.cci || c->npt != 8 || !c->d.lat || !c->d.pos2id || !c->have_family)
                return fail(PD_ERR_ARG, "pd_set_option: the tiled force needs a lattice, 2x2x2 points and a family");
            int* rad = reinterpret_cast<int*>(c->hscalar + 8);
            pd::launch_family_radius(c->d, reinterpret_cast<int*>(c->scal + pd::CG_NSLOT - 1), c->stream);
            PD_CUDA_TRY(cudaMemcpyAsync(rad, c->scal + pd::CG_NSLOT - 1, sizeof(int), cudaMemcpyDeviceToHost,
                                        c->stream));
            PD_CUDA_TRY(cudaStreamSynchronize(c->stream));
            pd::Dev t = c->d;
            t.fam_radius = *rad;
            t.tile_x = tx;
            t.tile_y = ty;
            t.tile_z = tz;
            const size_t smem = pd::tiled_smem_bytes(t);
            int dev = 0, optin = 0;
            PD_CUDA_TRY(cudaGetDevice(&dev));
            PD_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
            if (smem > (size_t)optin) return fail(PD_ERR_ARG, "pd_set_option: tile and halo exceed shared memory");
            if (pd::prepare_tiled_force(smem) != PD_OK) return fail(PD_ERR_CUDA, "pd_set_option: shared memory opt-in");
            c->d = t;
            break;
        }
        case PD_OPT_PERSIST_FORCE_CHUNK:
        case PD_OPT_PERSIST_GATHER_CHUNK:
            if (value < 128 || value > (1 << 20) || value % 128) return fail(PD_ERR_ARG, "pd_set_option: chunk");
            (option == PD_OPT_PERSIST_FORCE_CHUNK ? c->force_chunk : c->gather_chunk) = (unsigned)value;
            break;
        default: return fail(PD_ERR_ARG, "pd_set_option: unknown option");
    }
    c->generation++;  // captured graphs hold the old launch choice
    return PD_OK;
}

int pd_get_option(pd_ctx* c, int option, int64_t* value) {
    if (!c || !value) return fail(PD_ERR_ARG, "pd_get_option: null argument");
    switch (option) {
        case PD_OPT_F64_LANES_BELOW: *value = c->d.f64_lanes_below; return PD_OK;
        case PD_OPT_TILE: *value = c->tile; return PD_OK;
        case PD_OPT_PERSIST_BLOCKS_PER_SM: *value = c->persist_per_sm; return PD_OK;
        case PD_OPT_PERSIST_FORCE_CHUNK: *value = c->force_chunk; return PD_OK;
        case PD_OPT_PERSIST_GATHER_CHUNK: *value = c->gather_chunk; return PD_OK;
        case PD_OPT_STATIC_STENCIL: *value = c->static_stencil_opt; return PD_OK;
        case PD_OPT_STATIC_SPLIT: *value = c->static_split; return PD_OK;
        case PD_OPT_STATIC_F32_BELOW: *value = c->static_f32_below; return PD_OK;
        case PD_OPT_ADJOINT_VJP32: *value = c->adj_vjp32; return PD_OK;
        case PD_OPT_GATHER_PER_POINT: *value = c->d.gather_per_point; return PD_OK;
        case PD_OPT_FORCE_TILE:
            *value = c->d.tile_x | (c->d.tile_y << 8) | ((int64_t)c->d.tile_z << 16);
            return PD_OK;
        case PD_OPT_FORCE_QUAD: *value = c->d.force_quad; return PD_OK;
        case PD_OPT_GATHER_SELL: *value = c->d.sell_on; return PD_OK;
        case PD_OPT_FORCE_STENCIL: *value = c->fst_shape; return PD_OK;
        case PD_OPT_GATHER_STENCIL: *value = c->gpat_opt; return PD_OK;
        case PD_OPT_STATIC_PRECOND: *value = c->static_precond; return PD_OK;
        case PD_OPT_PERSIST_WAIT_US: *value = c->persist_wait_us; return PD_OK;
        case PD_OPT_PERSIST_TEST_STALL: *value = c->persist_stall; return PD_OK;
        default: return fail(PD_ERR_ARG, "pd_get_option: unknown option");
    }
}

int pd_set_energy(pd_ctx* c, int on) {
    if (!c) return fail(PD_ERR_ARG, "pd_set_energy: null context");
    c->d.energy = on ? 1 : 0;
    return PD_OK;
}

int pd_set_state(pd_ctx* c, const double* U, const double* V) {
    if (!c) return fail(PD_ERR_ARG, "pd_set_state: null context");
    const size_t b3 = sizeof(double) * 3 * c->n;
    if (U) {
        PD_TRY(upload_vec3(c, c->d.U, U));
        PD_CUDA_TRY(cudaMemcpyAsync(c->d.u1, c->d.U, b3, cudaMemcpyDeviceToDevice, c->stream));
        PD_CUDA_TRY(cudaMemcpyAsync(c->d.us, c->d.U, b3, cudaMemcpyDeviceToDevice, c->stream));
    }
    if (V) {
        PD_TRY(upload_vec3(c, c->d.V, V));
        PD_CUDA_TRY(cudaMemcpyAsync(c->d.vbuf, c->d.V, b3, cudaMemcpyDeviceToDevice, c->stream));
    }
    PD_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return PD_OK;
}

int pd_get_state(pd_ctx* c, double* U, double* V) {
    if (!c) return fail(PD_ERR_ARG, "pd_get_state: null context");
    if (U) PD_TRY(download_vec3(c, U, c->d.U));
    if (V) PD_TRY(download_vec3(c, V, c->d.V));
    return PD_OK;
}

int pd_get_vbuf(pd_ctx* c, double* vb) {
    if (!c || !vb) return fail(PD_ERR_ARG, "pd_get_vbuf: null argument");
    return download_vec3(c, vb, c->d.vbuf);
}

int pd_set_gauss_displ(pd_ctx* c, const double* ug) {
    if (!c || !ug) return fail(PD_ERR_ARG, "pd_set_gauss_displ: null argument");
    const int64_t M = c->n * c->npt;
    double* tmp = nullptr;
    PD_TRY(dalloc(c, &tmp, 3 * M));
    int rc = upload(c, tmp, ug, sizeof(double) * 3 * M);
    if (rc == PD_OK) {
        // [node][point][3] -> [point*3 + a][node]
        std::vector<double> h(3 * M);
        for (int64_t i = 0; i < c->n; ++i)
            for (int g = 0; g < c->npt; ++g)
                for (int a = 0; a < 3; ++a) h[(int64_t)(3 * g + a) * c->n + i] = ug[(i * c->npt + g) * 3 + a];
        rc = upload(c, c->d.ug, h.data(), sizeof(double) * 3 * M);
    }
    dfree(c, tmp);
    return rc;
}

int pd_get_gauss_displ(pd_ctx* c, double* ug) {
    if (!c || !ug) return fail(PD_ERR_ARG, "pd_get_gauss_displ: null argument");
    const int64_t M = c->n * c->npt;
    std::vector<double> h(3 * M);
    PD_CUDA_TRY(cudaMemcpyAsync(h.data(), c->d.ug, sizeof(double) * 3 * M, cudaMemcpyDeviceToHost, c->stream));
    PD_CUDA_TRY(cudaStreamSynchronize(c->stream));
    for (int64_t i = 0; i < c->n; ++i)
        for (int g = 0; g < c->npt; ++g)
            for (int a = 0; a < 3; ++a) ug[(i * c->npt + g) * 3 + a] = h[(int64_t)(3 * g + a) * c->n + i];
    return PD_OK;
}

int pd_get_energy_density(pd_ctx* c, double* eed) {
    if (!c || !eed) return fail(PD_ERR_ARG, "pd_get_energy_density: null argument");
    PD_CUDA_TRY(cudaMemcpyAsync(eed, c->d.eed, sizeof(double) * c->n, cudaMemcpyDeviceToHost, c->stream));
    PD_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return PD_OK;
}

int pd_init_dynamic(pd_ctx* c) {
    if (!c) return fail(PD_ERR_ARG, "pd_init_dynamic: null context");
    const size_t b3 = sizeof(double) * 3 * c->n;
    PD_CUDA_TRY(cudaMemcpyAsync(c->d.vbuf, c->d.V, b3, cudaMemcpyDeviceToDevice, c->stream));
    PD_CUDA_TRY(cudaMemsetAsync(c->d.eed, 0, sizeof(double) * c->n, c->stream));
    if (c->d.ai && c->have_ai) PD_CUDA_TRY(cudaMemsetAsync(c->d.ai_dmg, 0, sizeof(int32_t) * c->n, c->stream));
    PD_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return PD_OK;
}

int pd_gather(pd_ctx* c, double time, const double* us) {
    if (!c) return fail(PD_ERR_ARG, "pd_gather: null context");
    if (!ready_dynamic(c)) return fail(PD_ERR_ARG, "pd_gather: family/MLS data not set");
    PD_TRY(set_time(c, time));
    const double* src = c->d.U;
    if (us) {
        PD_TRY(upload_vec3(c, c->d.us, us));
        src = c->d.us;
    }
    if (c->precision == PD_PREC_FP32C) pd::launch_gather_f32c(c->d, src, c->stream);
    else pd::launch_gather_f64(c->d, src, c->stream);
    PD_CUDA_TRY(cudaGetLastError());
    PD_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return PD_OK;
}

int pd_force_stage(pd_ctx* c, double dt, double time, const double* us, double* k_out) {
    if (!c || !us) return fail(PD_ERR_ARG, "pd_force_stage: null argument");
    if (!ready_dynamic(c)) return fail(PD_ERR_ARG, "pd_force_stage: family/MLS data not set");
    PD_TRY(set_time(c, time));
    PD_TRY(upload_vec3(c, c->d.us, us));
    if (c->precision == PD_PREC_FP32C) pd::launch_force_f32c(c->d, dt, c->stream);
    else pd::launch_force_f64(c->d, dt, c->stream);
    pd::launch_epilogue(c->d, 0, dt, dt, c->stream);
    PD_CUDA_TRY(cudaGetLastError());
    if (k_out) PD_TRY(download_vec3(c, k_out, c->d.k1));
    PD_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return PD_OK;
}

int pd_rk4_step(pd_ctx* c, double dt, double time, double* ke, double* ee) {
    if (!c) return fail(PD_ERR_ARG, "pd_rk4_step: null context");
    if (!ready_dynamic(c)) return fail(PD_ERR_ARG, "pd_rk4_step: family/MLS data not set");
    PD_TRY(set_time(c, time));
    enqueue_step_body(c, dt);
    PD_CUDA_TRY(cudaGetLastError());
    if (c->d.energy && (ke || ee)) {
        PD_CUDA_TRY(cudaMemcpyAsync(c->hscalar, c->d.red + 2 * c->n, 2 * sizeof(double), cudaMemcpyDeviceToHost,
                                    c->stream));
    }
    PD_CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (ke) *ke = c->d.energy ? c->hscalar[0] : 0.0;
    if (ee) *ee = c->d.energy ? c->hscalar[1] : 0.0;
    return PD_OK;
}

int pd_rk4_steps(pd_ctx* c, double dt, double t0, int nsteps) {
    if (!c || nsteps < 0) return fail(PD_ERR_ARG, "pd_rk4_steps: bad argument");
    if (!ready_dynamic(c)) return fail(PD_ERR_ARG, "pd_rk4_steps: family/MLS data not set");
    if (nsteps == 0) return PD_OK;
    PD_TRY(set_time(c, t0));
    if (!c->step_graph || c->graph_dt != dt || c->graph_prec != c->precision || c->graph_energy != c->d.energy ||
        c->graph_generation != c->generation) {
        if (c->step_graph) {
            cudaGraphExecDestroy(c->step_graph);
            c->step_graph = nullptr;
        }
        cudaGraph_t g = nullptr;
        PD_CUDA_TRY(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        pd::launch_advance_time(c->d.tdev, dt, c->stream);
        enqueue_step_body(c, dt);
        cudaError_t e = cudaStreamEndCapture(c->stream, &g);
        if (e != cudaSuccess) return pd::fail_cuda(e, "capture", __FILE__, __LINE__);
        e = cudaGraphInstantiate(&c->step_graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return pd::fail_cuda(e, "instantiate", __FILE__, __LINE__);
        c->graph_dt = dt;
        c->graph_prec = c->precision;
        c->graph_energy = c->d.energy;
        c->graph_generation = c->generation;
    }
    for (int k = 0; k < nsteps; ++k) PD_CUDA_TRY(cudaGraphLaunch(c->step_graph, c->stream));
    PD_CUDA_TRY(cudaGetLastError());
    return PD_OK;
}

int pd_rk4_steps_host(pd_ctx* c, double dt, double t0, int nsteps, const double* U_in, const double* V_in,
                      double* U_out, double* V_out) {
    if (!c) return fail(PD_ERR_ARG, "pd_rk4_steps_host: null context");
    if (!ready_dynamic(c)) return fail(PD_ERR_ARG, "pd_rk4_steps_host: family/MLS data not set");
    const size_t b3 = sizeof(double) * 3 * c->n;
    if (U_in && c->n > 0) {
        // The first stage reads the Gauss-point displacements (and, in FP32C,
        // the node blocks) that the previous step's closing gather derived
        // from the device's U.  When the uploaded U differs from that U, they
        // are derived again from U_in at t0 (CalcIntgPointDisplRK4,
        // pdDataManager.cpp:2402-2495), so the steps start from U_in
        // throughout; a round trip of the device state skips the gather.
        PD_CUDA_TRY(cudaMemsetAsync(c->dflag, 0, sizeof(int), c->stream));
        PD_CUDA_TRY(cudaMemcpyAsync(c->scratch, U_in, b3, cudaMemcpyHostToDevice, c->stream));
        pd::launch_to_soa_changed(c->scratch, c->d.U, c->n, 3, c->dflag, c->stream);
        int* hflag = reinterpret_cast<int*>(c->hscalar + 12);
        PD_CUDA_TRY(cudaMemcpyAsync(hflag, c->dflag, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        PD_CUDA_TRY(cudaStreamSynchronize(c->stream));
        if (*hflag) {
            PD_TRY(set_time(c, t0));
            if (c->precision == PD_PREC_FP32C) pd::launch_gather_f32c(c->d, c->d.U, c->stream);
            else pd::launch_gather_f64(c->d, c->d.U, c->stream);
            PD_CUDA_TRY(cudaGetLastError());
        }
    }
    if (V_in) {
        PD_CUDA_TRY(cudaMemcpyAsync(c->scratch + 3 * c->n, V_in, b3, cudaMemcpyHostToDevice, c->stream));
        pd::launch_to_soa(c->scratch + 3 * c->n, c->d.V, c->n, 3, c->stream);
    }
    // nsteps - 1 steps from the step graph, the last one launched directly so
    // that U and V (final after its fourth stage) are copied out on a second
    // stream while its closing gather, which only reads U, runs
    if (nsteps > 1) PD_TRY(pd_rk4_steps(c, dt, t0, nsteps - 1));
    if (nsteps >= 1) {
        if (nsteps == 1) PD_TRY(set_time(c, t0));
        if (!c->copy_stream) {
            PD_CUDA_TRY(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
            PD_CUDA_TRY(cudaEventCreateWithFlags(&c->ev_final, cudaEventDisableTiming));
            PD_CUDA_TRY(cudaEventCreateWithFlags(&c->ev_copied, cudaEventDisableTiming));
        }
        pd::launch_advance_time(c->d.tdev, dt, c->stream);
        enqueue_step_body(c, dt, false);
        PD_CUDA_TRY(cudaEventRecord(c->ev_final, c->stream));
        PD_CUDA_TRY(cudaStreamWaitEvent(c->copy_stream, c->ev_final, 0));
        enqueue_closing_gather(c);
        cudaStream_t cs = c->copy_stream;
        if (U_out) {
            pd::launch_to_aos(c->d.U, c->scratch, c->n, 3, cs);
            PD_CUDA_TRY(cudaMemcpyAsync(U_out, c->scratch, b3, cudaMemcpyDeviceToHost, cs));
        }
        if (V_out) {
            pd::launch_to_aos(c->d.V, c->scratch + 3 * c->n, c->n, 3, cs);
            PD_CUDA_TRY(cudaMemcpyAsync(V_out, c->scratch + 3 * c->n, b3, cudaMemcpyDeviceToHost, cs));
        }
        // the next call's uploads into scratch wait for these copies
        PD_CUDA_TRY(cudaEventRecord(c->ev_copied, cs));
        PD_CUDA_TRY(cudaStreamWaitEvent(c->stream, c->ev_copied, 0));
        PD_CUDA_TRY(cudaGetLastError());
    } else {
        if (U_out) {
            pd::launch_to_aos(c->d.U, c->scratch, c->n, 3, c->stream);
            PD_CUDA_TRY(cudaMemcpyAsync(U_out, c->scratch, b3, cudaMemcpyDeviceToHost, c->stream));
        }
        if (V_out) {
            pd::launch_to_aos(c->d.V, c->scratch + 3 * c->n, c->n, 3, c->stream);
            PD_CUDA_TRY(cudaMemcpyAsync(V_out, c->scratch + 3 * c->n, b3, cudaMemcpyDeviceToHost, c->stream));
        }
    }
    PD_CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (c->copy_stream) PD_CUDA_TRY(cudaStreamSynchronize(c->copy_stream));
    return PD_OK;
}

int pd_reset_state(pd_ctx* c) {
    if (!c) return fail(PD_ERR_ARG, "pd_reset_state: null context");
    const size_t b3 = sizeof(double) * 3 * c->n;
    cudaStream_t s = c->stream;
    for (double* p : {c->d.U, c->d.V, c->d.vbuf, c->d.u1, c->d.us}) PD_CUDA_TRY(cudaMemsetAsync(p, 0, b3, s));
    PD_CUDA_TRY(cudaMemsetAsync(c->d.ug, 0, b3 * c->npt, s));
    PD_CUDA_TRY(cudaMemsetAsync(c->d.nblk, 0, sizeof(float) * c->n * c->d.bs, s));
    PD_CUDA_TRY(cudaMemsetAsync(c->d.eed, 0, sizeof(double) * c->n, s));
    if (c->d.ai && c->have_ai) {
        // the bonds the AI form broke heal: back to the family's own flags
        PD_CUDA_TRY(cudaMemcpyAsync(c->d.ai_brk, c->fbroken, c->H, cudaMemcpyDeviceToDevice, s));
        PD_CUDA_TRY(cudaMemsetAsync(c->d.ai_dmg, 0, sizeof(int32_t) * c->n, s));
    }
    PD_CUDA_TRY(cudaStreamSynchronize(s));
    return PD_OK;
}

int pd_profile_step(pd_ctx* c, double dt, double time, double* ms) {
    if (!c || !ms) return fail(PD_ERR_ARG, "pd_profile_step: null argument");
    if (!ready_dynamic(c)) return fail(PD_ERR_ARG, "pd_profile_step: family/MLS data not set");
    PD_TRY(set_time(c, time));
    cudaStream_t s = c->stream;
    const pd::Dev& d = c->d;
    const bool f32 = c->precision == PD_PREC_FP32C;
    const int64_t n3 = 3 * c->n;
    std::vector<cudaEvent_t> ev;
    std::vector<int> cls;
    auto mark = [&](int k) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        cudaEventRecord(e, s);
        ev.push_back(e);
        cls.push_back(k);
    };
    auto force = [&](double dts) {
        mark(-1);
        if (f32) pd::launch_force_f32c(d, dts, s);
        else pd::launch_force_f64(d, dts, s);
        mark(0);
    };
    auto gather = [&](const double* us) {
        mark(-1);
        if (f32) pd::launch_gather_f32c(d, us, s);
        else pd::launch_gather_f64(d, us, s);
        mark(1);
    };
    auto epi = [&](int st, double dts) {
        mark(-1);
        pd::launch_epilogue(d, st, dts, dt, s);
        mark(2);
    };
    const double h = 0.5 * dt;
    mark(-1);
    cudaMemcpyAsync(d.vbuf, d.V, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(d.u1, d.U, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(d.us, d.U, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s);
    if (d.energy) cudaMemsetAsync(d.eed, 0, sizeof(double) * c->n, s);
    mark(3);
    force(h); epi(1, h);
    gather(d.us); force(h); epi(2, h);
    gather(d.us); force(dt); epi(3, dt);
    gather(d.us); force(dt); epi(4, dt);
    mark(-1);
    if (d.energy) pd::launch_energy_reduce(d, s);
    mark(3);
    gather(d.U);
    cudaError_t e = cudaStreamSynchronize(s);
    for (int k = 0; k < 4; ++k) ms[k] = 0.0;
    for (size_t k = 1; k < ev.size(); ++k) {
        if (cls[k] < 0) continue;
        float t = 0.f;
        cudaEventElapsedTime(&t, ev[k - 1], ev[k]);
        ms[cls[k]] += t;
    }
    for (cudaEvent_t x : ev) cudaEventDestroy(x);
    if (e != cudaSuccess) return pd::fail_cuda(e, "profile step", __FILE__, __LINE__);
    return PD_OK;
}

int pd_evals_per_stage(pd_ctx* c, int64_t* ev) {
    if (!c || !ev) return fail(PD_ERR_ARG, "pd_evals_per_stage: null argument");
    if (!c->have_family) return fail(PD_ERR_ARG, "pd_evals_per_stage: no family");
    if (c->d.ai) {
        if (!c->have_ai) return fail(PD_ERR_ARG, "pd_evals_per_stage: no AI data");
        *ev = c->ai_points;  // trapezoid points of the unbroken bonds
        return PD_OK;
    }
    *ev = c->d.cci ? c->Ha : c->Ha * c->npt;
    return PD_OK;
}

// ----------------------------------------------------------------- static

}  // extern "C"

namespace {

// Decides once per setup whether the static operator can run as a stencil:
// every lattice position of a box holds one node, node id = x + nx (y + ny z),
// one material, no broken family entry, and every node's family is the union
// stencil clipped to the box (checked node by node on the downloaded family).
// The split form's tables (k_static_nd): the columns of the z-blocked
// difference form sorted by half-height, (w, w oz spacing) per oz, and the
// per-node diagonal blocks D_i built on the device from the same tables;
// the interior block is read back from a node at least the stencil reach
// inside the box.  Left off (ndcol = 0) beyond kNdMaxCol columns.
int split_prepare(pd_ctx* c, const std::vector<int4>& cols, const std::vector<double4>& colgeo) {
    pd::StencilDev& S = c->sten;
    S.ndcol = S.ndr = 0;
    const int nc = (int)cols.size(), rz = S.rz;
    if (nc == 0 || nc > pd::kNdMaxCol || rz < 1 || rz > 4) return PD_OK;
    const int W = 2 * rz + 1;
    std::vector<int> h(nc, 0), order(nc);
    for (int k = 0; k < nc; ++k) {
        for (int q = 0; q < W; ++q)
            if (colgeo[(size_t)k * W + q].w != 0.0) h[k] = std::max(h[k], std::abs(q - rz));
        order[k] = k;
    }
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return h[a] < h[b]; });
    std::vector<int4> nd(nc);
    std::vector<double2> tap((size_t)nc * 9, make_double2(0.0, 0.0));
    int rx = 0, ry = 0;
    for (int hh = 0; hh <= 5; ++hh) S.ndcls[hh] = nc;
    for (int k = nc - 1; k >= 0; --k) S.ndcls[h[order[k]]] = k;
    for (int hh = 4; hh >= 0; --hh) S.ndcls[hh] = std::min(S.ndcls[hh], S.ndcls[hh + 1]);
    for (int k = 0; k < nc; ++k) {
        const int o = order[k];
        nd[k] = make_int4(cols[o].x, cols[o].y, cols[o].z, h[o]);
        rx = std::max(rx, std::abs(cols[o].x));
        ry = std::max(ry, std::abs(cols[o].y));
        for (int q = 0; q < W; ++q) {
            const double4 g = colgeo[(size_t)o * W + q];
            tap[(size_t)k * 9 + 4 + (q - rz)] = make_double2(g.w, g.w * g.z);
        }
    }
    if (!c->nd_col) {
        PD_TRY(dalloc(c, &c->nd_col, pd::kMaxStencil));
        PD_TRY(dalloc(c, &c->nd_tap, (size_t)pd::kMaxStencil * 9));
    }
    if (!c->nd_diag) PD_TRY(dalloc(c, &c->nd_diag, (size_t)6 * c->n));
    PD_TRY(upload(c, c->nd_col, nd.data(), sizeof(int4) * nc));
    PD_TRY(upload(c, c->nd_tap, tap.data(), sizeof(double2) * tap.size()));
    S.ndcol = nc;
    S.nrx = rx;
    S.nry = ry;
    S.sp = c->d.dx;
    S.ndc = c->nd_col;
    S.ndtap = c->nd_tap;
    S.ndiag = c->nd_diag;
    if (!c->nd_host) c->nd_host.reset(new pd::NdTab());
    std::copy(tap.begin(), tap.end(), c->nd_host->tap);
    std::copy(nd.begin(), nd.end(), c->nd_host->col);
    S.ndhost = c->nd_host.get();
    pd::launch_static_ndiag(S, c->n, c->nd_diag, c->stream);
    PD_CUDA_TRY(cudaGetLastError());
    if (S.nx > 2 * rx && S.ny > 2 * ry && S.nz > 2 * rz) {
        const int64_t i = rx + (int64_t)S.nx * (ry + (int64_t)S.ny * rz);
        double* hv = c->hscalar;
        for (int k = 0; k < 6; ++k)
            PD_CUDA_TRY(cudaMemcpyAsync(hv + k, c->nd_diag + k * c->n + i, sizeof(double), cudaMemcpyDeviceToHost,
                                        c->stream));
        PD_CUDA_TRY(cudaStreamSynchronize(c->stream));
        for (int k = 0; k < 6; ++k) S.ndint[k] = hv[k];
        S.ndin = 1;
    } else {
        S.ndin = 0;  // no interior: every node reads its own block
    }
    S.ndr = c->static_split;
    return PD_OK;
}

int static_prepare(pd_ctx* c) {
    if (c->sten_gen == c->generation) return PD_OK;
    c->sten_ok = false;
    c->sten_gen = c->generation;
    if (!c->static_stencil_opt || c->d.multimat || c->d.nmat != 1 || c->n == 0) return PD_OK;
    const int64_t N = c->n;
    std::vector<int32_t> lat;
    if (!lattice_positions(c->coords, N, c->d.dx, lat)) return PD_OK;
    int64_t dims[3] = {0, 0, 0};
    for (int64_t i = 0; i < N; ++i) {
        dims[0] = std::max<int64_t>(dims[0], (lat[i] & 2047) + 1);
        dims[1] = std::max<int64_t>(dims[1], ((lat[i] >> 11) & 2047) + 1);
        dims[2] = std::max<int64_t>(dims[2], (lat[i] >> 22) + 1);
    }
    if (dims[0] * dims[1] * dims[2] != N) return PD_OK;
    for (int64_t i = 0; i < N; ++i) {
        const int64_t l = (lat[i] & 2047) + dims[0] * (((lat[i] >> 11) & 2047) + dims[1] * (lat[i] >> 22));
        if (l != i) return PD_OK;
    }
    if (c->Ha != c->H) return PD_OK;  // broken entries
    std::vector<int64_t> rp(N + 1);
    std::vector<int32_t> col(std::max<int64_t>(c->H, 1));
    PD_CUDA_TRY(cudaMemcpy(rp.data(), c->d.frow, sizeof(int64_t) * (N + 1), cudaMemcpyDeviceToHost));
    PD_CUDA_TRY(cudaMemcpy(col.data(), c->d.fcol, sizeof(int32_t) * c->H, cudaMemcpyDeviceToHost));
    const int64_t nx = dims[0], ny = dims[1], nz = dims[2];
    auto pos = [&](int64_t i, int64_t* q) {
        q[0] = i % nx;
        q[1] = (i / nx) % ny;
        q[2] = i / (nx * ny);
    };
    // union of the offsets, keyed (ox, oy, oz) in [-64, 63]^3
    std::vector<uint8_t> seen(128 * 128 * 128, 0);
    std::vector<std::array<int, 3>> offs;
    for (int64_t i = 0; i < N; ++i) {
        int64_t qi[3], qj[3];
        pos(i, qi);
        for (int64_t p = rp[i]; p < rp[i + 1]; ++p) {
            pos(col[p], qj);
            int o[3];
            for (int a = 0; a < 3; ++a) {
                o[a] = (int)(qj[a] - qi[a]);
                if (o[a] < -64 || o[a] > 63) return PD_OK;
            }
            const int key = ((o[0] + 64) << 14) | ((o[1] + 64) << 7) | (o[2] + 64);
            if (!seen[key]) {
                seen[key] = 1;
                offs.push_back({o[0], o[1], o[2]});
            }
        }
    }
    if (offs.empty() || offs.size() > (size_t)pd::kMaxStencil) return PD_OK;
    // every node's family has exactly the offsets that stay in the box
    for (int64_t i = 0; i < N; ++i) {
        int64_t qi[3];
        pos(i, qi);
        int64_t in = 0;
        for (const auto& o : offs)
            if (qi[0] + o[0] >= 0 && qi[0] + o[0] < nx && qi[1] + o[1] >= 0 && qi[1] + o[1] < ny &&
                qi[2] + o[2] >= 0 && qi[2] + o[2] < nz)
                ++in;
        if (in != rp[i + 1] - rp[i]) return PD_OK;
    }
    std::sort(offs.begin(), offs.end(), [&](const std::array<int, 3>& a, const std::array<int, 3>& b) {
        return a[0] + nx * (a[1] + ny * a[2]) < b[0] + nx * (b[1] + ny * b[2]);
    });
    const int ns = (int)offs.size();
    std::vector<int4> off(ns);
    std::vector<double4> geo(ns);
    const double h = c->d.dx, cv = c->mat_spring[0] * c->d.vol;
    int radius = 0;
    for (int k = 0; k < ns; ++k) {
        const auto& o = offs[k];
        off[k] = make_int4(o[0], o[1], o[2], (int)(o[0] + nx * (o[1] + ny * o[2])));
        const double e0 = o[0] * h, e1 = o[1] * h, e2 = o[2] * h;
        const double r2 = e0 * e0 + e1 * e1 + e2 * e2, r = std::sqrt(r2);
        geo[k] = make_double4(e0, e1, e2, cv / (r2 * r));
        for (int a = 0; a < 3; ++a) radius = std::max(radius, std::abs(o[a]));
    }
    // the same stencil by (ox, oy) columns with a dense oz window (the
    // z-blocked kernel), when no offset reaches beyond 4 along z
    int rz = 0;
    for (const auto& o : offs) rz = std::max(rz, std::abs(o[2]));
    std::vector<int4> cols;
    std::vector<double4> colgeo;
    if (rz >= 1 && rz <= 4) {
        const int W = 2 * rz + 1;
        std::map<std::pair<int, int>, int> at;  // (oy, ox) -> column
        for (int k = 0; k < ns; ++k) {
            const auto key = std::make_pair(offs[k][1], offs[k][0]);
            if (!at.count(key)) at[key] = 0;
        }
        int nc = 0;
        for (auto& kv : at) {
            kv.second = nc++;
            cols.push_back(make_int4(kv.first.second, kv.first.first, (int)(kv.first.second + nx * kv.first.first), 0));
        }
        colgeo.assign((size_t)nc * W, make_double4(0.0, 0.0, 0.0, 0.0));
        for (int k = 0; k < ns; ++k) {
            const int cidx = at[std::make_pair(offs[k][1], offs[k][0])];
            colgeo[(size_t)cidx * W + offs[k][2] + rz] = geo[k];
        }
    }
    if (!c->sten_off) {
        PD_TRY(dalloc(c, &c->sten_off, pd::kMaxStencil));
        PD_TRY(dalloc(c, &c->sten_geo, pd::kMaxStencil));
        PD_TRY(dalloc(c, &c->sten_pmask, N));
        PD_TRY(dalloc(c, &c->sten_xm, 3 * N));
        PD_TRY(dalloc(c, &c->sten_col, pd::kMaxStencil));
        PD_TRY(dalloc(c, &c->sten_colgeo, (size_t)pd::kMaxStencil * 9));
    }
    PD_TRY(upload(c, c->sten_off, off.data(), sizeof(int4) * ns));
    PD_TRY(upload(c, c->sten_geo, geo.data(), sizeof(double4) * ns));
    if (!cols.empty() && cols.size() <= (size_t)pd::kMaxStencil && colgeo.size() <= (size_t)pd::kMaxStencil * 9) {
        PD_TRY(upload(c, c->sten_col, cols.data(), sizeof(int4) * cols.size()));
        PD_TRY(upload(c, c->sten_colgeo, colgeo.data(), sizeof(double4) * colgeo.size()));
    } else {
        cols.clear();
    }
    pd::launch_static_pmask(c->d, c->sten_pmask, c->stream);
    PD_CUDA_TRY(cudaStreamSynchronize(c->stream));
    c->sten = pd::StencilDev{(int)nx, (int)ny, (int)nz, ns, radius, c->sten_off, c->sten_geo, c->sten_pmask,
                             c->sten_xm, (int)cols.size(), rz, c->sten_col, c->sten_colgeo};
    PD_TRY(split_prepare(c, cols, colgeo));
    c->sten_ok = true;
    return PD_OK;
}

// y = K x: the stencil kernel when static_prepare accepted the problem, the
// family-list kernel otherwise; f32: FP32 bond terms on FP64 vectors
void static_apply(pd_ctx* c, double time, bool f32, const double* x, double* y) {
    if (c->sten_ok) pd::launch_static_stencil(c->d, c->sten, f32, x, y, c->stream);
    else if (f32) pd::launch_static_apply_f32x(c->d, time, x, y, c->stream);
    else pd::launch_static_apply_f64(c->d, time, x, y, c->stream);
}

}  // namespace

extern "C" {

int pd_static_prepare(pd_ctx* c, int* stencil) {
    if (!c) return fail(PD_ERR_ARG, "pd_static_prepare: null context");
    if (!c->have_family) return fail(PD_ERR_ARG, "pd_static_prepare: no family");
    PD_TRY(static_prepare(c));
    if (stencil) *stencil = c->sten_ok ? 1 : 0;
    return PD_OK;
}

int pd_static_matvec(pd_ctx* c, double time, const double* x, double* y) {
    if (!c || !x || !y) return fail(PD_ERR_ARG, "pd_static_matvec: null argument");
    if (!c->have_family) return fail(PD_ERR_ARG, "pd_static_matvec: no family");
    PD_TRY(static_prepare(c));
    PD_TRY(upload_vec3(c, c->d.us, x));
    static_apply(c, time, false, c->d.us, c->d.k1);
    PD_CUDA_TRY(cudaGetLastError());
    return download_vec3(c, y, c->d.k1);
}

int pd_static_rhs(pd_ctx* c, double time, double* b) {
    if (!c || !b) return fail(PD_ERR_ARG, "pd_static_rhs: null argument");
    if (!c->have_family) return fail(PD_ERR_ARG, "pd_static_rhs: no family");
    pd::launch_static_rhs(c->d, time, c->d.k1, c->stream);
    PD_CUDA_TRY(cudaGetLastError());
    return download_vec3(c, b, c->d.k1);
}

}  // extern "C"

namespace {

// Preconditioned CG on K x = b with FP64 vectors and device scalars; the
// residual is read back every 10 iterations.  minv: the block-Jacobi
// preconditioner (3x3 diagonal blocks, k_static_bjacobi), or null for plain
// CG.  f32: once the relative residual is below f32_below, the matvec of the
// iterations has FP32 bond terms, and the residual is replaced by the FP64
// true residual b - K x whenever the recurred one has fallen by 1e-2 since
// the last replacement and when it reaches the tolerance ("reliable
// updates", van der Vorst & Ye, SIAM J. Sci. Comput. 22 (2000) 1716-1731):
// the FP64 refinement of the FP32 iterations, without restarting the Krylov
// space.  The first iterations stay FP64 because rounding errors there cost
// the most: on block-Jacobi CG of clamped lattice cubes, FP32 matvecs from
// the start took 1.2-1.5x the FP64 iteration count, FP32 matvecs only below
// a relative residual of 0.1 took the FP64 count (inexact Krylov methods
// tolerate matvec errors that grow as the residual falls: Simoncini & Szyld,
// SIAM J. Sci. Comput. 25 (2003) 454-477).  Convergence is decided on the
// true residual.  scal: CG_RR = r.z, CG_RRN = the next r.z, CG_RES = r.r.
int cg_static(pd_ctx* c, double time, const double* b, double* x, double* r, double* p, double* q, double* z,
              const double* minv, bool f32, double f32_below, double rtol, int maxit, int* iters, double* relres,
              int* replacements) {
    const int64_t n3 = 3 * c->n;
    cudaStream_t s = c->stream;
    double* scal = c->scal;
    auto dot = [&](const double* a, const double* bb, double* out) {
        pd::launch_dot_f64(a, bb, n3, c->dotpart, out, s);
    };
    auto read = [&]() -> int {
        PD_CUDA_TRY(cudaGetLastError());
        PD_CUDA_TRY(cudaMemcpyAsync(c->hscalar, scal, sizeof(double) * 5, cudaMemcpyDeviceToHost, s));
        PD_CUDA_TRY(cudaStreamSynchronize(s));
        return PD_OK;
    };
    // z = M^-1 r (z aliases r without a preconditioner) and r.z into slot
    const double* zz = minv ? z : r;
    auto precond = [&](double* slot) {
        if (minv) pd::launch_bj_apply(minv, r, z, c->n, s);
        dot(r, zz, slot);
    };
    // true residual into r, |r|^2 into scal[CG_RES], r.z into scal[CG_RR]
    auto true_residual = [&]() {
        static_apply(c, time, false, x, q);
        pd::launch_sub_f64(b, q, r, n3, s);
        dot(r, r, scal + pd::CG_RES);
        precond(scal + pd::CG_RR);
    };
    dot(b, b, scal + pd::CG_BB);
    true_residual();
    PD_CUDA_TRY(cudaMemcpyAsync(p, zz, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s));
    PD_TRY(read());
    const double bb = c->hscalar[pd::CG_BB] > 0.0 ? c->hscalar[pd::CG_BB] : 1.0;
    double rel = std::sqrt(c->hscalar[pd::CG_RES] / bb);
    double since = rel;  // largest recurred residual since the last replacement
    int it = 0, nrep = 0;
    const int check = 10;
    while (rel > rtol && it < maxit) {
        const bool use32 = f32 && rel < f32_below;
        for (int k = 0; k < check && it < maxit; ++k, ++it) {
            static_apply(c, time, use32, p, q);
            dot(p, q, scal + pd::CG_PQ);
            pd::launch_cg_update_x_f64(x, r, p, q, n3, scal, s);
            precond(scal + pd::CG_RRN);
            pd::launch_cg_update_p_f64(zz, p, n3, scal, s);
            pd::launch_cg_swap(scal, s);
        }
        dot(r, r, scal + pd::CG_RES);
        PD_TRY(read());
        rel = std::sqrt(c->hscalar[pd::CG_RES] / bb);
        if (!std::isfinite(rel)) break;
        since = std::max(since, rel);
        if (f32 && (rel <= rtol || rel < 1e-2 * since)) {
            // replace: r = b - K x in FP64; p keeps its direction
            true_residual();
            PD_TRY(read());
            rel = std::sqrt(c->hscalar[pd::CG_RES] / bb);
            since = rel;
            ++nrep;
        }
    }
    if (iters) *iters = it;
    if (relres) *relres = rel;
    if (replacements) *replacements = nrep;
    return (rel <= rtol) ? PD_OK : PD_ERR_NOCONV;
}

}  // namespace

// Matrix-free CG on the static system (replaces the dense Gauss-Jordan of
// pdSolve::Gauss, pdSolve.cpp:545-673).
extern "C" int pd_static_solve(pd_ctx* c, double time, int precision, double rtol, int maxit, double* x, int* iters,
                               double* relres) {
    if (!c || !x) return fail(PD_ERR_ARG, "pd_static_solve: null argument");
    if (!c->have_family) return fail(PD_ERR_ARG, "pd_static_solve: no family");
    if (precision != PD_PREC_FP64 && precision != PD_PREC_FP64A && precision != PD_PREC_FP32C)
        return fail(PD_ERR_ARG, "pd_static_solve: precision");
    PD_TRY(static_prepare(c));
    const int64_t n3 = 3 * c->n;
    double *b = nullptr, *xd = nullptr, *r = nullptr, *p = nullptr, *q = nullptr, *z = nullptr;
    PD_TRY(dalloc(c, &b, n3));
    PD_TRY(dalloc(c, &xd, n3));
    PD_TRY(dalloc(c, &r, n3));
    PD_TRY(dalloc(c, &p, n3));
    PD_TRY(dalloc(c, &q, n3));
    if (c->static_precond) PD_TRY(dalloc(c, &z, n3));
    auto cleanup = [&]() { dfree(c, b); dfree(c, xd); dfree(c, r); dfree(c, p); dfree(c, q); dfree(c, z); };
    int rc = upload_vec3(c, xd, x);
    if (rc != PD_OK) { cleanup(); return rc; }
    if (c->static_precond && (!c->bj_minv || c->bj_gen != c->generation)) {
        if (!c->bj_minv && (rc = dalloc(c, &c->bj_minv, (size_t)(6 * c->n))) != PD_OK) { cleanup(); return rc; }
        pd::launch_static_bjacobi(c->d, c->bj_minv, c->stream);
        c->bj_gen = c->generation;
    }
    pd::launch_static_rhs(c->d, time, b, c->stream);
    int it = 0, nrep = 0;
    double rel = 0.0;
    rc = cg_static(c, time, b, xd, r, p, q, z, c->static_precond ? c->bj_minv : nullptr,
                   precision == PD_PREC_FP32C, c->static_f32_below > 0 ? 1.0 / c->static_f32_below : 2.0, rtol,
                   maxit, &it, &rel, &nrep);
    c->static_replacements = nrep;
    int rc2 = download_vec3(c, x, xd);
    cleanup();
    if (iters) *iters = it;
    if (relres) *relres = rel;
    if (rc == PD_ERR_NOCONV) return fail(PD_ERR_NOCONV, "static solve did not reach the tolerance");
    return rc != PD_OK ? rc : rc2;
}

// ---------------------------------------------------------------- adjoint

extern "C" int pd_set_spring_factor(pd_ctx* c, const double* f) {
    if (!c || !f) return fail(PD_ERR_ARG, "pd_set_spring_factor: null argument");
    for (int64_t i = 0; i < c->n; ++i)
        if (!(f[i] > 0.0) || !std::isfinite(f[i])) return fail(PD_ERR_ARG, "pd_set_spring_factor: factors must be positive");
    if (!c->d.sfac) {
        double* sf = nullptr;
        PD_TRY(dalloc(c, &sf, c->n));
        c->d.sfac = sf;
    }
    PD_TRY(upload(c, (void*)c->d.sfac, f, sizeof(double) * c->n));
    c->sfac_host.assign(f, f + c->n);
    c->generation++;
    return upload_static_f32(c);
}

namespace {

// one RK4 step (as enqueue_step_body) that copies, before every force
// evaluation, the state the force reads: U, the trial displacement and the
// Gauss-point displacements (tape[s] = {U, us, ug} of stage s; in the FP32
// form ug is rebuilt in FP64 from the node blocks the force reads)
void enqueue_step_tape(pd_ctx* c, double dt, double* tape, bool f32) {
    cudaStream_t s = c->stream;
    const pd::Dev& d = c->d;
    const int64_t n3 = 3 * c->n, ng = n3 * c->npt;
    const int64_t per = 2 * n3 + ng;
    auto copy = [&](int st) {
        double* t = tape + (int64_t)(st - 1) * per;
        cudaMemcpyAsync(t, d.U, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(t + n3, d.us, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s);
        if (f32) pd::launch_blocks_to_ug(d, t + 2 * n3, s);
        else cudaMemcpyAsync(t + 2 * n3, d.ug, sizeof(double) * ng, cudaMemcpyDeviceToDevice, s);
    };
    auto force = [&](double dts) {
        if (f32) pd::launch_force_f32c(d, dts, s);
        else pd::launch_force_f64(d, dts, s);
    };
    auto gather = [&](const double* us) {
        if (f32) pd::launch_gather_f32c(d, us, s);
        else pd::launch_gather_f64(d, us, s);
    };
    const double h = 0.5 * dt;
    pd::launch_advance_time(d.tdev, dt, s);
    cudaMemcpyAsync(d.vbuf, d.V, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(d.u1, d.U, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(d.us, d.U, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s);
    copy(1);
    force(h);
    pd::launch_epilogue(d, 1, h, dt, s);
    gather(d.us);
    copy(2);
    force(h);
    pd::launch_epilogue(d, 2, h, dt, s);
    gather(d.us);
    copy(3);
    force(dt);
    pd::launch_epilogue(d, 3, dt, dt, s);
    gather(d.us);
    copy(4);
    force(dt);
    pd::launch_epilogue(d, 4, dt, dt, s);
    gather(d.U);
}

// transpose of the contributor lists of nodes without a boundary condition
int build_transpose(pd_ctx* c) {
    if (c->tptr) return PD_OK;
    const int64_t N = c->n;
    std::vector<int64_t> cnt(N + 1, 0);
    for (int64_t j = 0; j < N; ++j) {
        if (c->bc_host[j] >= 0) continue;
        for (int64_t p = c->cbptr_host[j]; p < c->cbptr_host[j + 1]; ++p) cnt[c->cbidx_host[p] + 1]++;
    }
    for (int64_t k = 0; k < N; ++k) cnt[k + 1] += cnt[k];
    std::vector<int64_t> fill(cnt.begin(), cnt.end() - 1);
    std::vector<int32_t> tj(std::max<int64_t>(cnt[N], 1)), tpos(std::max<int64_t>(cnt[N], 1));
    for (int64_t j = 0; j < N; ++j) {
        if (c->bc_host[j] >= 0) continue;
        for (int64_t p = c->cbptr_host[j]; p < c->cbptr_host[j + 1]; ++p) {
            const int64_t k = c->cbidx_host[p];
            tj[fill[k]] = (int32_t)j;
            tpos[fill[k]] = (int32_t)(p - c->cbptr_host[j]);
            fill[k]++;
        }
    }
    PD_TRY(dalloc(c, &c->tptr, N + 1));
    PD_TRY(dalloc(c, &c->tj, tj.size()));
    PD_TRY(dalloc(c, &c->tpos, tpos.size()));
    PD_TRY(upload(c, c->tptr, cnt.data(), sizeof(int64_t) * (N + 1)));
    PD_TRY(upload(c, c->tj, tj.data(), sizeof(int32_t) * tj.size()));
    PD_TRY(upload(c, c->tpos, tpos.data(), sizeof(int32_t) * tpos.size()));
    return PD_OK;
}

void free_checkpoints(pd_ctx* c) {
    for (auto& k : c->ckpt) {
        dfree(c, k.U);
        dfree(c, k.V);
        dfree(c, k.ug);
        dfree(c, k.blk);
    }
    c->ckpt.clear();
}

int save_checkpoint(pd_ctx* c, pd_ctx::Checkpoint& k) {
    const int64_t n3 = 3 * c->n, ng = n3 * c->npt;
    if (!k.U) {
        PD_TRY(dalloc(c, &k.U, n3));
        PD_TRY(dalloc(c, &k.V, n3));
        PD_TRY(dalloc(c, &k.ug, ng));
    }
    cudaStream_t s = c->stream;
    PD_CUDA_TRY(cudaMemcpyAsync(k.U, c->d.U, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s));
    PD_CUDA_TRY(cudaMemcpyAsync(k.V, c->d.V, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s));
    PD_CUDA_TRY(cudaMemcpyAsync(k.ug, c->d.ug, sizeof(double) * ng, cudaMemcpyDeviceToDevice, s));
    if (c->adj_f32) {
        const size_t nb = (size_t)c->n * c->d.bs;
        if (!k.blk) PD_TRY(dalloc(c, &k.blk, nb));
        PD_CUDA_TRY(cudaMemcpyAsync(k.blk, c->d.nblk, sizeof(float) * nb, cudaMemcpyDeviceToDevice, s));
    }
    PD_CUDA_TRY(cudaMemcpyAsync(c->hscalar, c->d.tdev, sizeof(double), cudaMemcpyDeviceToHost, s));
    PD_CUDA_TRY(cudaStreamSynchronize(s));
    k.t = c->hscalar[0];
    return PD_OK;
}

}  // namespace

// Forward run of nsteps RK4 steps from the current state, keeping a
// checkpoint (U, V, Gauss-point u, time) every checkpoint_every steps for
// pd_adjoint_backward.  PD_PREC_FP64A stays FP64A and PD_PREC_FP32C stays
// FP32C (its checkpoints also keep the node blocks the next step reads);
// PD_PREC_FP64 runs as PD_PREC_FP64.
extern "C" int pd_adjoint_forward(pd_ctx* c, double dt, double t0, int nsteps, int every) {
    if (!c || nsteps < 1 || every < 1) return fail(PD_ERR_ARG, "pd_adjoint_forward: bad argument");
    if (!ready_dynamic(c)) return fail(PD_ERR_ARG, "pd_adjoint_forward: family/MLS data not set");
    if (c->d.cci || c->d.ai)
        return fail(PD_ERR_ARG, "pd_adjoint_forward: the adjoint covers the Gauss-point (FGI) scheme");
    const int prec = c->precision, energy = c->d.energy;
    if (prec != PD_PREC_FP64A && prec != PD_PREC_FP32C) c->precision = PD_PREC_FP64;
    c->adj_acc = c->d.acc_stretch = prec == PD_PREC_FP64A;
    c->adj_f32 = prec == PD_PREC_FP32C;
    c->d.energy = 0;
    free_checkpoints(c);
    const int nck = (nsteps + every - 1) / every;
    c->ckpt.resize(nck);
    int rc = set_time(c, t0);
    int done = 0;
    for (int k = 0; k < nck && rc == PD_OK; ++k) {
        rc = save_checkpoint(c, c->ckpt[k]);
        if (rc != PD_OK) break;
        const int n = std::min(every, nsteps - done);
        rc = pd_rk4_steps(c, dt, c->ckpt[k].t, n);
        done += n;
    }
    if (rc == PD_OK) {
        cudaError_t e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) rc = pd::fail_cuda(e, "adjoint forward", __FILE__, __LINE__);
    }
    c->precision = prec;
    c->d.energy = energy;
    c->adj_steps = rc == PD_OK ? nsteps : 0;
    c->adj_every = every;
    c->adj_dt = dt;
    return rc;
}

// Reverse sweep of the last pd_adjoint_forward.  lam_U, lam_V: adjoints of
// the final U and V ([3N] host, V may be NULL); grad_f [N] receives the
// gradient with respect to the per-node spring factors.  Leaves the state
// at the start of the forward run.
extern "C" int pd_adjoint_backward(pd_ctx* c, const double* lam_U, const double* lam_V, double* grad_f) {
    if (!c || !lam_U || !grad_f) return fail(PD_ERR_ARG, "pd_adjoint_backward: null argument");
    if (c->adj_steps < 1) return fail(PD_ERR_ARG, "pd_adjoint_backward: no forward run to reverse");
    if (!c->d.sfac) return fail(PD_ERR_ARG, "pd_adjoint_backward: set the spring factors first");
    if (c->d.mls) PD_TRY(build_transpose(c));
    const int64_t N = c->n, n3 = 3 * N, ng = n3 * c->npt;
    cudaStream_t s = c->stream;
    const pd::Dev& d = c->d;
    const double dt = c->adj_dt;
    // work buffers: carved from one pool that the context keeps between calls
    // (an optimiser calls the pair again and again with the same sizes)
    const int64_t pool_need = 13 * n3 + 3 * ng + N + (int64_t)c->adj_every * 4 * (2 * n3 + ng) + 32 * 19;
    if (c->adj_pool_count < pool_need) {
        dfree(c, c->adj_pool);
        c->adj_pool = nullptr;
        c->adj_pool_count = 0;
        if (dalloc(c, &c->adj_pool, pool_need) != PD_OK)
            return fail(PD_ERR_OOM, "pd_adjoint_backward: device memory for the tape");
        c->adj_pool_count = pool_need;
    }
    int64_t carved = 0;
    auto get = [&](int64_t count) -> double* {
        double* p = c->adj_pool + carved;
        carved += (count + 31) / 32 * 32;  // 256-byte aligned pieces
        return carved <= c->adj_pool_count ? p : nullptr;
    };
    pd::AdjBuf A;
    double** fields[] = {&A.lU, &A.lV, &A.lvb, &A.lu1, &A.lk1, &A.lk2, &A.lk3, &A.lk4, &A.lus, &A.lF, &A.lueff};
    bool ok = true;
    for (double** f : fields) ok = ok && ((*f = get(n3)) != nullptr);
    double* lUp = get(n3);
    double* lVp = get(n3);
    double* lugSp = get(ng);
    double* lug = get(ng);
    double* lugSn = get(ng);
    double* gradf = get(N);
    const int every = c->adj_every;
    const int64_t per = 2 * n3 + ng;
    double* tape = get((int64_t)every * 4 * per);
    auto release = [&]() {};
    if (!ok || !lUp || !lVp || !lugSp || !lug || !lugSn || !gradf || !tape) {
        release();
        return fail(PD_ERR_OOM, "pd_adjoint_backward: device memory for the tape");
    }
    const int energy = c->d.energy, acc = c->d.acc_stretch;
    const bool f32 = c->adj_f32, vjp32 = f32 && c->adj_vjp32;
    c->d.energy = 0;  // the recomputed steps need no energy density
    c->d.acc_stretch = c->adj_acc;  // and use the forward run's arithmetic
    int rc = upload_vec3(c, lUp, lam_U);
    if (rc == PD_OK && lam_V) rc = upload_vec3(c, lVp, lam_V);
    if (rc == PD_OK && !lam_V) rc = cudaMemsetAsync(lVp, 0, sizeof(double) * n3, s) == cudaSuccess ? PD_OK : PD_ERR_CUDA;
    cudaMemsetAsync(lugSp, 0, sizeof(double) * ng, s);
    cudaMemsetAsync(gradf, 0, sizeof(double) * N, s);
    const int nck = (int)c->ckpt.size();
    for (int k = nck - 1; k >= 0 && rc == PD_OK; --k) {
        const pd_ctx::Checkpoint& K = c->ckpt[k];
        const int S = std::min(every, c->adj_steps - k * every);
        // restore the segment's start and recompute it with the stage tape
        cudaMemcpyAsync(d.U, K.U, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(d.V, K.V, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(d.ug, K.ug, sizeof(double) * ng, cudaMemcpyDeviceToDevice, s);
        rc = set_time(c, K.t);
        if (f32)  // the node blocks the segment started from
            cudaMemcpyAsync(d.nblk, K.blk, sizeof(float) * (size_t)N * d.bs, cudaMemcpyDeviceToDevice, s);
        for (int n = 0; n < S && rc == PD_OK; ++n) enqueue_step_tape(c, dt, tape + (int64_t)n * 4 * per, f32);
        // reverse the segment's steps
        for (int n = S - 1; n >= 0 && rc == PD_OK; --n) {
            const double* tp = tape + (int64_t)n * 4 * per;
            auto teU = [&](int st) { return tp + (int64_t)(st - 1) * per; };
            auto teus = [&](int st) { return tp + (int64_t)(st - 1) * per + n3; };
            auto teug = [&](int st) { return tp + (int64_t)(st - 1) * per + 2 * n3; };
            pd::launch_gather_T(d, c->tptr, c->tj, c->tpos, lugSp, lUp, s);
            pd::launch_adj_combine(d, dt, lUp, lVp, A, s);
            double* lk_of[5] = {nullptr, A.lk1, A.lk2, A.lk3, A.lk4};
            const double alpha[5] = {0.0, 0.0, 0.5, 0.5, 1.0};
            for (int st = 4; st >= 2; --st) {
                const double dts = st >= 3 ? dt : 0.5 * dt;
                pd::launch_adj_stage_pre(d, dts, lk_of[st], A, s);
                pd::launch_vjp_own(d, teU(st), teus(st), teug(st), A.lF, A.lueff, gradf, s, vjp32);
                pd::launch_vjp_partner(d, teU(st), teus(st), teug(st), A.lF, lug, gradf, s, vjp32);
                pd::launch_adj_stage_node(d, A, s);
                pd::launch_gather_T(d, c->tptr, c->tj, c->tpos, lug, A.lus, s);
                pd::launch_adj_stage_post(d, alpha[st], lk_of[st - 1], A, s);
            }
            pd::launch_adj_stage_pre(d, 0.5 * dt, A.lk1, A, s);
            pd::launch_vjp_own(d, teU(1), teus(1), teug(1), A.lF, A.lueff, gradf, s, vjp32);
            pd::launch_vjp_partner(d, teU(1), teus(1), teug(1), A.lF, lugSn, gradf, s, vjp32);
            pd::launch_adj_stage1_end(d, A, s);
            cudaMemcpyAsync(lUp, A.lU, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s);
            cudaMemcpyAsync(lVp, A.lV, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s);
            std::swap(lugSp, lugSn);
            cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) rc = pd::fail_cuda(e, "adjoint step", __FILE__, __LINE__);
        }
    }
    if (rc == PD_OK) {
        // leave the state at the start of the forward run
        const pd_ctx::Checkpoint& K = c->ckpt[0];
        cudaMemcpyAsync(d.U, K.U, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(d.V, K.V, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(d.ug, K.ug, sizeof(double) * ng, cudaMemcpyDeviceToDevice, s);
        if (f32) cudaMemcpyAsync(d.nblk, K.blk, sizeof(float) * (size_t)N * d.bs, cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(grad_f, gradf, sizeof(double) * N, cudaMemcpyDeviceToHost, s);
        cudaError_t e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) rc = pd::fail_cuda(e, "adjoint backward", __FILE__, __LINE__);
    }
    release();
    c->d.energy = energy;
    c->d.acc_stretch = acc;
    return rc;
}

// ------------------------------------------------------- persistent stepping

namespace {

bool persist_capable(const pd_ctx* c) {
    return c->precision == PD_PREC_FP32C && !c->d.cci && c->npt == 8 && c->d.gc_host && !c->d.energy;
}

int persist_blocks(pd_ctx* c, int* blocks) {
    int per_sm = 0, sms = 0;
    if (pd::persist_max_blocks(c->d, &per_sm, &sms) != PD_OK || per_sm < 1)
        return fail(PD_ERR_CUDA, "persistent launch: no cooperative launch of this kernel fits the device");
    const int use = c->persist_per_sm > 0 ? std::min(c->persist_per_sm, per_sm) : per_sm;
    *blocks = use * sms;
    return PD_OK;
}

}  // namespace

// nsteps RK4 steps of the FP32-compensated FGI form (2x2x2 points) in one
// cooperative persistent launch: work-queue phases separated by bounded grid
// barriers.  The control-block reset and the launch are captured once into a
// CUDA graph (per dt, step count and launch shape) and replayed.  Same
// result bit for bit as pd_rk4_steps in PD_PREC_FP32C.  Synchronous: the
// call waits for the launch and reports a barrier that gave up as
// PD_ERR_TIMEOUT.
extern "C" int pd_rk4_steps_persistent(pd_ctx* c, double dt, double t0, int nsteps) {
    if (!c || nsteps < 0) return fail(PD_ERR_ARG, "pd_rk4_steps_persistent: bad argument");
    if (!ready_dynamic(c)) return fail(PD_ERR_ARG, "pd_rk4_steps_persistent: family/MLS data not set");
    if (!persist_capable(c))
        return fail(PD_ERR_ARG,
                    "pd_rk4_steps_persistent: needs PD_PREC_FP32C, Gauss-point integration with 2x2x2 points and "
                    "energy accumulation off");
    if (nsteps == 0) return PD_OK;
    const size_t bytes = sizeof(pd::PersistCtl) + sizeof(unsigned) * 8 * (size_t)nsteps;
    if (c->pctl_steps < nsteps) {
        if (c->persist_graph) {
            cudaGraphExecDestroy(c->persist_graph);
            c->persist_graph = nullptr;
        }
        dfree(c, c->pctl);
        c->pctl = nullptr;
        c->pctl_steps = 0;
        char* p = nullptr;
        PD_TRY(dalloc(c, &p, bytes));
        c->pctl = (pd::PersistCtl*)p;
        c->pctl_steps = nsteps;
    }
    int blocks = 0;
    PD_TRY(persist_blocks(c, &blocks));
    PD_TRY(set_time(c, t0));
    if (!c->persist_graph || c->persist_dt != dt || c->persist_steps != nsteps ||
        c->persist_generation != c->generation) {
        if (c->persist_graph) {
            cudaGraphExecDestroy(c->persist_graph);
            c->persist_graph = nullptr;
        }
        cudaGraph_t g = nullptr;
        PD_CUDA_TRY(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        cudaError_t e = cudaMemsetAsync(c->pctl, 0, bytes, c->stream);
        if (e == cudaSuccess)
            e = pd::launch_persist_f32c(c->d, dt, nsteps, c->pctl, blocks, c->force_chunk, c->gather_chunk,
                                        pd::PersistWait{(unsigned long long)c->persist_wait_us * 1000ull,
                                                        c->persist_stall},
                                        c->stream);
        cudaError_t e2 = cudaStreamEndCapture(c->stream, &g);
        if (e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return pd::fail_cuda(e, "persistent launch capture", __FILE__, __LINE__);
        }
        if (e2 != cudaSuccess) return pd::fail_cuda(e2, "persistent launch capture", __FILE__, __LINE__);
        e = cudaGraphInstantiate(&c->persist_graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return pd::fail_cuda(e, "persistent graph instantiate", __FILE__, __LINE__);
        c->persist_dt = dt;
        c->persist_steps = nsteps;
        c->persist_generation = c->generation;
    }
    PD_CUDA_TRY(cudaGraphLaunch(c->persist_graph, c->stream));
    PD_CUDA_TRY(cudaMemcpyAsync(c->hscalar, &c->pctl->error, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    PD_CUDA_TRY(cudaStreamSynchronize(c->stream));
    int err = 0;
    std::memcpy(&err, c->hscalar, sizeof(int));
    if (err) return fail(PD_ERR_TIMEOUT, "pd_rk4_steps_persistent: a grid barrier gave up waiting");
    return PD_OK;
}

// ---------------------------------------------------------------- autotuner

namespace {

struct Snapshot {
    double *U = nullptr, *V = nullptr, *ug = nullptr, t = 0.0;
    float* nblk = nullptr;
};

int snap_take(pd_ctx* c, Snapshot& S) {
    const int64_t n3 = 3 * c->n, ng = n3 * c->npt, nb = c->n * (int64_t)c->d.bs;
    cudaStream_t s = c->stream;
    if (!S.U) {
        PD_TRY(dalloc(c, &S.U, n3));
        PD_TRY(dalloc(c, &S.V, n3));
        PD_TRY(dalloc(c, &S.ug, ng));
        PD_TRY(dalloc(c, &S.nblk, nb));
    }
    PD_CUDA_TRY(cudaMemcpyAsync(S.U, c->d.U, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s));
    PD_CUDA_TRY(cudaMemcpyAsync(S.V, c->d.V, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s));
    PD_CUDA_TRY(cudaMemcpyAsync(S.ug, c->d.ug, sizeof(double) * ng, cudaMemcpyDeviceToDevice, s));
    PD_CUDA_TRY(cudaMemcpyAsync(S.nblk, c->d.nblk, sizeof(float) * nb, cudaMemcpyDeviceToDevice, s));
    PD_CUDA_TRY(cudaMemcpyAsync(c->hscalar, c->d.tdev, sizeof(double), cudaMemcpyDeviceToHost, s));
    PD_CUDA_TRY(cudaStreamSynchronize(s));
    S.t = c->hscalar[0];
    return PD_OK;
}

int snap_restore(pd_ctx* c, const Snapshot& S) {
    const int64_t n3 = 3 * c->n, ng = n3 * c->npt, nb = c->n * (int64_t)c->d.bs;
    cudaStream_t s = c->stream;
    PD_CUDA_TRY(cudaMemcpyAsync(c->d.U, S.U, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s));
    PD_CUDA_TRY(cudaMemcpyAsync(c->d.V, S.V, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s));
    PD_CUDA_TRY(cudaMemcpyAsync(c->d.ug, S.ug, sizeof(double) * ng, cudaMemcpyDeviceToDevice, s));
    PD_CUDA_TRY(cudaMemcpyAsync(c->d.nblk, S.nblk, sizeof(float) * nb, cudaMemcpyDeviceToDevice, s));
    PD_TRY(set_time(c, S.t));
    PD_CUDA_TRY(cudaStreamSynchronize(s));
    return PD_OK;
}

void snap_free(pd_ctx* c, Snapshot& S) {
    dfree(c, S.U);
    dfree(c, S.V);
    dfree(c, S.ug);
    dfree(c, S.nblk);
}

// device time of `steps` steps from the snapshot, after an untimed run of
// the same length (which captures the graphs)
int time_steps(pd_ctx* c, const Snapshot& S, double dt, int steps, bool persistent, double* ms) {
    PD_TRY(snap_restore(c, S));
    if (persistent) PD_TRY(pd_rk4_steps_persistent(c, dt, S.t, steps));
    else PD_TRY(pd_rk4_steps(c, dt, S.t, steps));
    PD_TRY(snap_restore(c, S));
    cudaEvent_t a, b;
    PD_CUDA_TRY(cudaEventCreate(&a));
    PD_CUDA_TRY(cudaEventCreate(&b));
    cudaEventRecord(a, c->stream);
    int rc = persistent ? pd_rk4_steps_persistent(c, dt, S.t, steps) : pd_rk4_steps(c, dt, S.t, steps);
    cudaEventRecord(b, c->stream);
    cudaError_t e = cudaEventSynchronize(b);
    float f = 0.f;
    if (rc == PD_OK && e == cudaSuccess) cudaEventElapsedTime(&f, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (rc != PD_OK) return rc;
    if (e != cudaSuccess) return pd::fail_cuda(e, "autotune timing", __FILE__, __LINE__);
    *ms = f / steps;
    return PD_OK;
}

}  // namespace

// Times candidate launch shapes on this context's own problem and keeps the
// fastest: first the node-order tile with the graph-captured step, then the
// FP32 gather and force variants, then (when the persistent launch applies)
// its blocks per SM and queue chunk sizes.
// The state is restored after every trial, so tuning leaves it as it was.
extern "C" int pd_autotune(pd_ctx* c, double dt, int steps, pd_tune_result* out) {
    if (!c || !out || steps < 1 || !(dt > 0.0)) return fail(PD_ERR_ARG, "pd_autotune: bad argument");
    if (!ready_dynamic(c)) return fail(PD_ERR_ARG, "pd_autotune: family/MLS data not set");
    std::memset(out, 0, sizeof *out);
    Snapshot S;
    int rc = snap_take(c, S);
    auto done = [&](int r) {
        snap_free(c, S);
        return r;
    };
    if (rc != PD_OK) return done(rc);
    struct Trial {
        int64_t tile;
        int persistent, per_sm;
        unsigned fc, gc;
        double ms;
    };
    Trial best{c->tile, 0, c->persist_per_sm, c->force_chunk, c->gather_chunk, 1e300};
    auto apply = [&](const Trial& T) -> int {
        if (T.tile != c->tile) PD_TRY(pd_set_option(c, PD_OPT_TILE, T.tile));
        c->persist_per_sm = T.per_sm;
        c->force_chunk = T.fc;
        c->gather_chunk = T.gc;
        c->generation++;
        return PD_OK;
    };
    auto trial = [&](Trial T) -> int {
        PD_TRY(apply(T));
        PD_TRY(time_steps(c, S, dt, steps, T.persistent != 0, &T.ms));
        out->trials++;
        if (T.ms < best.ms) best = T;
        return PD_OK;
    };
    // tiles: only meaningful on a lattice
    std::vector<int64_t> tiles = {c->tile};
    if (c->d.lat) {
        const int64_t cand[][3] = {{3, 2, 2}, {3, 3, 1}, {4, 2, 1}, {2, 2, 2}, {4, 1, 1}, {3, 1, 1}, {5, 1, 0}};
        tiles.clear();
        for (auto& t3 : cand) tiles.push_back(t3[0] | (t3[1] << 8) | (t3[2] << 16));
    }
    for (int64_t tl : tiles)
        if ((rc = trial({tl, 0, c->persist_per_sm, c->force_chunk, c->gather_chunk, 0.0})) != PD_OK) return done(rc);
    if (c->precision == PD_PREC_FP32C && c->d.mls) {
        // the gather variant, on the best tile so far
        const int gp0 = c->d.gather_per_point;
        const double before = best.ms;
        c->d.gather_per_point = !gp0;
        Trial T{best.tile, 0, c->persist_per_sm, c->force_chunk, c->gather_chunk, 0.0};
        if ((rc = trial(T)) != PD_OK) return done(rc);
        if (!(best.ms < before)) c->d.gather_per_point = gp0;
        out->gather_per_point = c->d.gather_per_point;
        if (c->npt == 8 && !c->d.gather_per_point) {
            // every combination of the SELL copy (rebuilt for every later order
            // trial) and the contributor patterns (refused when nothing
            // repeats); both together run the coefficient ring
            const int s0 = c->d.sell_on, p0 = c->gpat_opt;
            int ks = s0, kp = p0;
            for (int sv = 0; sv <= 1; ++sv)
                for (int pv = 0; pv <= 1; ++pv) {
                    if (sv == s0 && pv == p0) continue;  // the shape timed so far
                    if ((rc = pd_set_option(c, PD_OPT_GATHER_SELL, sv)) != PD_OK) return done(rc);
                    if (pd_set_option(c, PD_OPT_GATHER_STENCIL, pv) != PD_OK) continue;
                    const double prev = best.ms;
                    Trial T2{best.tile, 0, c->persist_per_sm, c->force_chunk, c->gather_chunk, 0.0};
                    if ((rc = trial(T2)) != PD_OK) return done(rc);
                    if (best.ms < prev) {
                        ks = sv;
                        kp = pv;
                    }
                }
            if ((rc = pd_set_option(c, PD_OPT_GATHER_SELL, ks)) != PD_OK) return done(rc);
            if ((rc = pd_set_option(c, PD_OPT_GATHER_STENCIL, kp)) != PD_OK) return done(rc);
        }
        out->gather_sell = c->d.sell_on;
        out->gather_stencil = c->gpat_opt;
    }
    if (c->precision == PD_PREC_FP32C && !c->d.cci && c->npt == 8 && c->d.lat && !c->d.multimat) {
        // the lattice-stencil force in each block shape, on the best shape so far
        const int f0 = c->fst_shape;
        int keep = f0;
        const double before = best.ms;
        for (int sh = 1; sh <= 4; ++sh) {
            if (pd_set_option(c, PD_OPT_FORCE_STENCIL, sh) != PD_OK) break;  // not a box lattice: skip
            Trial T{best.tile, 0, c->persist_per_sm, c->force_chunk, c->gather_chunk, 0.0};
            const double prev = best.ms;
            if ((rc = trial(T)) != PD_OK) return done(rc);
            if (best.ms < prev) keep = sh;
        }
        if ((rc = pd_set_option(c, PD_OPT_FORCE_STENCIL, best.ms < before ? keep : f0)) != PD_OK) return done(rc);
        out->force_stencil = c->fst_shape;
    }
    if (c->precision == PD_PREC_FP32C && !c->d.cci && c->npt == 8 && c->d.lat && !c->d.hasfail &&
        !c->d.multimat && !c->fst_shape) {
        // four nodes per thread in the force, on the best shape so far
        const double before = best.ms;
        c->d.force_quad = 1;
        Trial T{best.tile, 0, c->persist_per_sm, c->force_chunk, c->gather_chunk, 0.0};
        if ((rc = trial(T)) != PD_OK) return done(rc);
        if (!(best.ms < before)) c->d.force_quad = 0;
        c->generation++;
        out->force_quad = c->d.force_quad;
    }
    if (c->precision == PD_PREC_FP32C && !c->d.cci && c->npt == 8 && c->d.lat && c->d.pos2id &&
        !c->d.force_quad && !c->fst_shape) {
        // the shared-memory tiles of the force, on the best shape so far
        const int tz = std::min(c->d.lat_nz, 4);
        const int64_t cand[][3] = {{16, 8, tz}, {32, 4, tz}, {16, 4, tz}, {8, 8, tz}, {32, 8, tz}, {64, 2, tz}};
        int64_t keep = 0;
        const double before = best.ms;
        for (auto& t3 : cand) {
            const int64_t v = t3[0] | (t3[1] << 8) | (t3[2] << 16);
            if (pd_set_option(c, PD_OPT_FORCE_TILE, v) != PD_OK) continue;  // does not fit: skip
            Trial T{best.tile, 0, c->persist_per_sm, c->force_chunk, c->gather_chunk, 0.0};
            const double prev = best.ms;
            if ((rc = trial(T)) != PD_OK) return done(rc);
            if (best.ms < prev) keep = v;
        }
        if ((rc = pd_set_option(c, PD_OPT_FORCE_TILE, best.ms < before ? keep : 0)) != PD_OK) return done(rc);
        out->force_tile = c->d.tile_x | (c->d.tile_y << 8) | ((int64_t)c->d.tile_z << 16);
    }
    if (persist_capable(c)) {
        int per_sm = 0, sms = 0;
        if (pd::persist_max_blocks(c->d, &per_sm, &sms) == PD_OK && per_sm >= 1) {
            const int64_t tl = best.tile;
            for (int ps = per_sm; ps >= 1 && ps >= per_sm - 2; --ps)
                for (unsigned fc : {128u, 512u})
                    for (unsigned gcn : {256u, 1024u})
                        if ((rc = trial({tl, 1, ps, fc, gcn, 0.0})) != PD_OK) return done(rc);
        }
    }
    if ((rc = apply(best)) != PD_OK) return done(rc);
    if ((rc = snap_restore(c, S)) != PD_OK) return done(rc);
    out->tile = best.tile;
    out->persistent = best.persistent;
    out->blocks_per_sm = best.per_sm;
    out->force_chunk = (int32_t)best.fc;
    out->gather_chunk = (int32_t)best.gc;
    out->ms_per_step = best.ms;
    c->tuned_persistent = best.persistent;
    return done(PD_OK);
}
