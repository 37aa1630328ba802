// C ABI of the host layer (include/pdmtel_host.h).
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "pdDataManager.h"
#include "pdmtel_host.h"

struct pdh_model {
    pdh::pdDataManager dat;
    std::string err;
};

namespace {
int track(pdh_model* m, int rc) {
    if (rc != PD_OK) m->err = m->dat.LastError();
    return rc;
}
}  // namespace

extern "C" {

int pdh_open(const char* dir, pdh_model** out) {
    if (!dir || !out) return PD_ERR_ARG;
    *out = nullptr;
    pdh_model* m = new (std::nothrow) pdh_model();
    if (!m) return PD_ERR_OOM;
    int rc = m->dat.SetWkDir(dir);
    if (rc == PD_OK) rc = m->dat.ReadInputFile();
    if (rc != PD_OK) m->err = m->dat.LastError();
    *out = m;  // kept even on error so that pdh_last_error can report it
    return rc;
}

int pdh_batch_create(const char* out_dir, pdh_model* const* specimens, int count, pdh_model** out) {
    if (!out_dir || !specimens || count < 1 || !out) return PD_ERR_ARG;
    *out = nullptr;
    pdh_model* m = new (std::nothrow) pdh_model();
    if (!m) return PD_ERR_OOM;
    std::vector<pdh::pdDataManager*> sp;
    for (int k = 0; k < count; ++k) {
        if (!specimens[k]) {
            m->err = "pdh_batch_create: null specimen";
            *out = m;
            return PD_ERR_ARG;
        }
        sp.push_back(&specimens[k]->dat);
    }
    int rc = m->dat.SetOutputDir(out_dir);
    if (rc == PD_OK) rc = m->dat.InitBatch(sp);
    if (rc != PD_OK) m->err = m->dat.LastError();
    *out = m;
    return rc;
}

int pdh_batch_offsets(pdh_model* m, int64_t* offsets) {
    if (!m || !offsets) return PD_ERR_ARG;
    if (!m->dat.IsBatch()) {
        m->err = "pdh_batch_offsets: not a batch model";
        return PD_ERR_ARG;
    }
    const std::vector<int64_t>& o = m->dat.BatchOffsets();
    std::memcpy(offsets, o.data(), sizeof(int64_t) * o.size());
    return PD_OK;
}

int pdh_batch_count(pdh_model* m, int* count) {
    if (!m || !count) return PD_ERR_ARG;
    *count = m->dat.IsBatch() ? (int)m->dat.BatchOffsets().size() - 1 : 0;
    return PD_OK;
}

int pdh_close(pdh_model* m) {
    delete m;
    return PD_OK;
}

const char* pdh_last_error(pdh_model* m) { return m ? m->err.c_str() : "null model"; }

int pdh_get_info(pdh_model* m, pdh_info* I) {
    if (!m || !I) return PD_ERR_ARG;
    std::memset(I, 0, sizeof *I);
    pdh::pdDataManager& d = m->dat;
    I->num_nodes = d.GetNumNode();
    I->num_halves = d.GetNumHalves();
    I->num_broken = d.GetNumBroken();
    I->num_contrib = d.NumContrib();
    I->num_gauss = d.GetNumGaussPoints();
    I->cci = d.IsCCI();
    I->mls = d.IsMLSOn();
    I->bdry_eff_on = 0;
    for (int a = 0; a < 3; ++a) I->dims[a] = d.GetGridDimension(a);
    I->total_step = d.GetTotalStep();
    I->dump_frequency = d.GetStepDumpFrequency();
    I->num_max_family = d.GetNumMaxFamily();
    I->grid_spacing = d.GetGridSpacing();
    I->horizon = d.GetHorizon();
    I->total_time = d.GetTotalTime();
    I->stable_dt = d.CalcStableTimeStep();
    I->min_bond_length = d.GetMinBondLength();
    I->ke = d.GetKinetTotal();
    I->ee = d.GetElastStep();
    I->num_materials = (int32_t)d.Materials().size();
    I->num_bcs = (int32_t)d.BCs().size();
    I->intg_point = d.GetIntgPoint();
    I->damping = d.GetDamping();
    return PD_OK;
}

int pdh_get_tables(pdh_model* m, pd_material* materials, pd_bc* bcs, double* abscissae, double* weights) {
    if (!m) return PD_ERR_ARG;
    std::vector<pd_material> mt;
    std::vector<pd_bc> bt;
    m->dat.DeviceTables(mt, bt);
    if (materials) std::memcpy(materials, mt.data(), sizeof(pd_material) * mt.size());
    if (bcs) std::memcpy(bcs, bt.data(), sizeof(pd_bc) * bt.size());
    const std::vector<double>& a = m->dat.GaussAbscissae();
    const std::vector<double>& w = m->dat.GaussWeights();
    if (abscissae) std::memcpy(abscissae, a.data(), sizeof(double) * a.size());
    if (weights) std::memcpy(weights, w.data(), sizeof(double) * w.size());
    return PD_OK;
}

int pdh_init_node(pdh_model* m) { return m ? track(m, m->dat.InitNode()) : PD_ERR_ARG; }
int pdh_init_bond(pdh_model* m) { return m ? track(m, m->dat.InitBond()) : PD_ERR_ARG; }
int pdh_init_material(pdh_model* m) { return m ? track(m, m->dat.InitMaterial()) : PD_ERR_ARG; }
int pdh_init_bdry_effect_factor(pdh_model* m) { return m ? track(m, m->dat.InitBdryEffectFactor()) : PD_ERR_ARG; }
int pdh_init_grid_boundary(pdh_model* m) { return m ? track(m, m->dat.InitGridBoundary()) : PD_ERR_ARG; }
int pdh_init_integration_point(pdh_model* m) { return m ? track(m, m->dat.InitIntegrationPoint()) : PD_ERR_ARG; }

int pdh_initial_problem(pdh_model* m) {
    if (!m) return PD_ERR_ARG;
    int rc;
    if ((rc = track(m, m->dat.InitNode())) != PD_OK) return rc;
    if ((rc = track(m, m->dat.InitBond())) != PD_OK) return rc;
    if ((rc = track(m, m->dat.InitMaterial())) != PD_OK) return rc;
    if ((rc = track(m, m->dat.InitBdryEffectFactor())) != PD_OK) return rc;
    if ((rc = track(m, m->dat.InitGridBoundary())) != PD_OK) return rc;
    return track(m, m->dat.InitIntegrationPoint());
}

int pdh_set_family(pdh_model* m, const int64_t* rp, const int32_t* col, const uint8_t* broken, double min_bond) {
    if (!m || !rp) return PD_ERR_ARG;
    const int64_t n = m->dat.GetNumNode();
    const int64_t H = rp[n];
    std::vector<int64_t> r(rp, rp + n + 1);
    std::vector<int32_t> c(col, col + H);
    std::vector<uint8_t> b;
    if (broken) b.assign(broken, broken + H);
    return track(m, m->dat.SetFamily(r, c, b, min_bond));
}

int pdh_set_spring_factor(pdh_model* m, const double* f) {
    if (!m || !f) return PD_ERR_ARG;
    if (m->dat.Context()) {
        m->err = "pdh_set_spring_factor: must precede the first GPU call";
        return PD_ERR_ARG;
    }
    m->dat.SetSpringFactor(std::vector<double>(f, f + m->dat.GetNumNode()));
    return PD_OK;
}

int pdh_get_nodes(pdh_model* m, double* x, int32_t* mat, int32_t* bc) {
    if (!m) return PD_ERR_ARG;
    const auto& d = m->dat;
    if (x) std::memcpy(x, d.Coords().data(), sizeof(double) * d.Coords().size());
    if (mat) std::memcpy(mat, d.MatIds().data(), sizeof(int32_t) * d.MatIds().size());
    if (bc) std::memcpy(bc, d.BcIds().data(), sizeof(int32_t) * d.BcIds().size());
    return PD_OK;
}

int pdh_get_family(pdh_model* m, int64_t* rp, int32_t* col, uint8_t* broken) {
    if (!m) return PD_ERR_ARG;
    const auto& d = m->dat;
    if (rp) std::memcpy(rp, d.FamilyPtr().data(), sizeof(int64_t) * d.FamilyPtr().size());
    if (col) std::memcpy(col, d.FamilyCol().data(), sizeof(int32_t) * d.FamilyCol().size());
    if (broken) std::memcpy(broken, d.FamilyBroken().data(), d.FamilyBroken().size());
    return PD_OK;
}

int pdh_get_bdry_eff(pdh_model* m, double* bE) {
    if (!m || !bE) return PD_ERR_ARG;
    std::memcpy(bE, m->dat.BdryEff().data(), sizeof(double) * m->dat.BdryEff().size());
    return PD_OK;
}

int pdh_get_mls(pdh_model* m, int64_t* cp, int32_t* ci, double* co) {
    if (!m) return PD_ERR_ARG;
    const int rc = track(m, m->dat.FetchMLS());
    if (rc != PD_OK) return rc;
    const auto& d = m->dat;
    if (cp) std::memcpy(cp, d.ContribPtr().data(), sizeof(int64_t) * d.ContribPtr().size());
    if (ci) std::memcpy(ci, d.ContribIdx().data(), sizeof(int32_t) * d.ContribIdx().size());
    if (co) std::memcpy(co, d.Coeff().data(), sizeof(double) * d.Coeff().size());
    return PD_OK;
}

int pdh_context(pdh_model* m, pd_ctx** ctx) {
    if (!m || !ctx) return PD_ERR_ARG;
    int rc = track(m, m->dat.InitDynamicSolve());
    *ctx = m->dat.Context();
    return rc;
}

int pdh_set_precision(pdh_model* m, int p) { return m ? track(m, m->dat.SetPrecision(p)) : PD_ERR_ARG; }

int pdh_post_afd(pdh_model* m, int step, int n, const int32_t* kind, const int32_t* norm, const double* coord,
                 const int64_t* node) {
    if (!m || n < 0 || (n > 0 && (!kind || !norm || !coord || !node))) return PD_ERR_ARG;
    std::vector<pdh::pdSolve::AfdRequest> req((size_t)n);
    for (int k = 0; k < n; ++k) req[k] = {kind[k], norm[k], coord[k], node[k]};
    return track(m, pdh::pdSolve::PostAFD(m->dat, step, req));
}

int pdh_set_device_setup(pdh_model* m, int on) {
    if (!m) return PD_ERR_ARG;
    m->dat.SetDeviceSetup(on != 0);
    return PD_OK;
}

int pdh_solve_dynamic(pdh_model* m, int write_files) {
    return m ? track(m, pdh::pdSolve::SolveDynamic(m->dat, write_files != 0)) : PD_ERR_ARG;
}

int pdh_solve_static(pdh_model* m, int precision, double rtol, int* iters, double* relres) {
    if (!m) return PD_ERR_ARG;
    std::vector<double> u(3 * (size_t)m->dat.GetNumNode(), 0.0);
    int rc = track(m, m->dat.StaticSolve(m->dat.CalcStableTimeStep(), precision, rtol, 200000, u, iters, relres));
    if (rc != PD_OK) return rc;
    std::vector<double> V(u.size(), 0.0);
    return track(m, m->dat.SetState(u, V));
}

}  // extern "C"
