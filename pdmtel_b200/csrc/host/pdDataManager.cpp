// pdDataManager / pdSolve of the drop-in (see pdDataManager.h).
#include "pdDataManager.h"

#include <algorithm>
#include <unordered_map>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <array>
#include <sstream>
#include <thread>

#include "pd_deck.h"

namespace pdh {

namespace {
const double kPI = std::acos(-1.0);  // pdIntgManager.h:25

enum { DISPL = 1, VELOC, DISPLGRAD, TRACTION };

int host_threads() {
    unsigned n = std::thread::hardware_concurrency();
    if (const char* e = std::getenv("PDMTEL_HOST_THREADS")) n = (unsigned)std::max(1, std::atoi(e));
    return (int)std::max(1u, std::min(n, 64u));
}
}  // namespace

pdDataManager::pdDataManager() {}

pdDataManager::~pdDataManager() {
    if (_ctx) pd_ctx_destroy(_ctx);
}

int pdDataManager::Error(int code, const std::string& msg) {
    _err = msg;
    if (!_outFilePath.empty()) {
        std::ofstream o(_outFilePath.c_str(), std::ios::app);
        o << msg << "\n";
    }
    return code;
}

int pdDataManager::Cuda(int rc, const char* what) {
    if (rc == PD_OK) return rc;
    return Error(rc, std::string(what) + ": " + pd_last_error());
}

int pdDataManager::SetWkDir(const std::string& dir) {
    _workDir = dir;
    if (!_workDir.empty() && _workDir.back() != '/') _workDir += '/';
    _inFilePath = _workDir + "pds_input.txt";
    _outFilePath = _workDir + "pds_output.dat";
    std::ifstream in(_inFilePath.c_str());
    if (!in) return Error(PD_ERR_ARG, "SetWkDir: input file not exits! " + _inFilePath);
    std::ofstream out(_outFilePath.c_str(), std::ios::out);
    return PD_OK;
}

int pdDataManager::SetOutputDir(const std::string& dir) {
    _workDir = dir;
    if (!_workDir.empty() && _workDir.back() != '/') _workDir += '/';
    _inFilePath.clear();
    _outFilePath = _workDir + "pds_output.dat";
    std::ofstream out(_outFilePath.c_str(), std::ios::out);
    if (!out) return Error(PD_ERR_ARG, "SetOutputDir: cannot write " + _outFilePath);
    return PD_OK;
}

// pdDataManager::ReadInputFile, pdDataManager.cpp:4-758
int pdDataManager::ReadInputFile() {
    DeckReader D;
    if (!D.Load(_inFilePath)) return Error(PD_ERR_ARG, "ReadInputFile: cannot open " + _inFilePath);
    std::ofstream log(_outFilePath.c_str(), std::ios::app);
    auto req = [&](const std::string& k) -> int {
        if (!D.Find(k)) return Error(PD_ERR_ARG, "FindKeyword: required keyword " + k + " not found!");
        return PD_OK;
    };
    int rc;
    auto rd = [&](const std::string& k, int pos, auto& v) -> int {
        int e = D.Read(k, pos, v);
        if (e == 1) return Error(PD_ERR_ARG, "ReadKeyword: keyword not found, keyword = " + k);
        if (e == 2) return Error(PD_ERR_ARG, "ReadKeyword: value missing at desired position, keyword = " + k);
        return PD_OK;
    };
#define PDH_TRY(x)                          \
    do {                                    \
        if ((rc = (x)) != PD_OK) return rc; \
    } while (0)
    _title = "Peridynamic test problem";
    if (D.Find("problem_title")) PDH_TRY(rd("problem_title", 1, _title));
    for (int a = 0; a < 3; ++a) _center[a] = 0.0;
    if (D.Find("grid_center"))
        for (int a = 0; a < 3; ++a) PDH_TRY(rd("grid_center", a + 1, _center[a]));
    PDH_TRY(req("grid_dimension"));
    for (int a = 0; a < 3; ++a) PDH_TRY(rd("grid_dimension", a + 1, _dims[a]));
    PDH_TRY(req("grid_spacing"));
    PDH_TRY(rd("grid_spacing", 1, _gridSpacing));
    if (D.Find("horizon")) PDH_TRY(rd("horizon", 1, _horizon));
    else _horizon = 3.015 * _gridSpacing;
    PDH_TRY(req("total_time"));
    PDH_TRY(rd("total_time", 1, _totalTime));
    PDH_TRY(req("total_step"));
    PDH_TRY(rd("total_step", 1, _totalStep));
    PDH_TRY(req("step_dump_frequency"));
    PDH_TRY(rd("step_dump_frequency", 1, _stepDumpFrequency));
    _safeFactor = 0.8;
    if (D.Find("safety_factor")) PDH_TRY(rd("safety_factor", 1, _safeFactor));
    _fixedTimeStepOn = false;
    if (D.Find("fixed_time_step")) {
        _fixedTimeStepOn = true;
        PDH_TRY(rd("fixed_time_step", 1, _fixedTimeStep));
    }
    if (D.Find("grid_file")) return Error(PD_ERR_ARG, "ReadInputFile: external grid files are not supported");
    _forcePlaneOn = D.Find("total_force_plane");
    if (_forcePlaneOn)
        for (int a = 0; a < 3; ++a) PDH_TRY(rd("total_force_plane", a + 1, _forcePlane[a]));
    // materials
    PDH_TRY(req("number_of_materials"));
    int nm = 0;
    PDH_TRY(rd("number_of_materials", 1, nm));
    if (nm <= 0) return Error(PD_ERR_ARG, "ReadInputFile: number_of_materials must be positive");
    _mats.assign(nm, Material());
    for (int i = 0; i < nm; ++i) {
        const std::string k = keyword_append("material_", i + 1);
        Material& m = _mats[i];
        PDH_TRY(rd(k, 1, m.type));
        if (m.type == 1) {
            PDH_TRY(rd(k, 2, m.ymod));
            PDH_TRY(rd(k, 3, m.sigmay));
            PDH_TRY(rd(k, 4, m.ecrit));
            PDH_TRY(rd(k, 5, m.density));
            m.nu = 0.25;  // pdMaterialBond.cpp:10
        } else if (m.type == 2) {
            PDH_TRY(rd(k, 2, m.ymod));
            PDH_TRY(rd(k, 3, m.sigmay));
            PDH_TRY(rd(k, 4, m.nu));
            PDH_TRY(rd(k, 5, m.ecrit));
            PDH_TRY(rd(k, 6, m.density));
        } else {
            return Error(PD_ERR_ARG, "ReadInputFile: unknown material type in " + k);
        }
        const std::string gk = keyword_append("gravity_", i + 1);
        if (D.Find(gk))
            for (int a = 0; a < 3; ++a) PDH_TRY(rd(gk, a + 1, m.grav[a]));
    }
    // boundary conditions
    PDH_TRY(req("number_of_boundary_conditions"));
    int nb = 0;
    PDH_TRY(rd("number_of_boundary_conditions", 1, nb));
    _bcs.assign(std::max(nb, 0), BdryCondition());
    for (int i = 0; i < nb; ++i) {
        const std::string k = keyword_append("boundary_condition_", i + 1);
        BdryCondition& b = _bcs[i];
        PDH_TRY(rd(k, 1, b.type));
        if (b.type < DISPL || b.type > TRACTION) return Error(PD_ERR_ARG, "ReadInputFile: unknown bc type in " + k);
        for (int a = 0; a < 3; ++a) PDH_TRY(rd(k, a + 2, b.dir[a]));
        const int nv = b.type == DISPLGRAD ? 9 : 3;
        b.value.assign(nv, 0.0);
        for (int a = 0; a < nv; ++a) PDH_TRY(rd(k, a + 5, b.value[a]));
        PDH_TRY(rd(k, nv + 5, b.end_time));
        PDH_TRY(rd(k, nv + 6, b.load_type));
    }
    // spaces
    auto read_space = [&](const std::string& k, bool has_ref, int nref, Space& s) -> int {
        int r;
        if ((r = rd(k, 1, s.geo)) != PD_OK) return r;
        int pos = 2;
        if (has_ref) {
            int id = 0;
            if ((r = rd(k, pos++, id)) != PD_OK) return r;
            s.ref = id - 1;
            if (s.ref < 0 || s.ref >= nref) return Error(PD_ERR_ARG, "ReadInputFile: id out of range in " + k);
        }
        if (s.geo == 1) {
            for (int a = 0; a < 3; ++a) {
                if ((r = rd(k, pos++, s.lo[a])) != PD_OK) return r;
                if ((r = rd(k, pos++, s.hi[a])) != PD_OK) return r;
            }
        } else if (s.geo == 2) {
            if ((r = rd(k, pos++, s.rad)) != PD_OK) return r;
            if ((r = rd(k, pos++, s.c1)) != PD_OK) return r;
            if ((r = rd(k, pos++, s.c2)) != PD_OK) return r;
            if ((r = rd(k, pos++, s.lo[2])) != PD_OK) return r;
            if ((r = rd(k, pos++, s.hi[2])) != PD_OK) return r;
        } else {
            return Error(PD_ERR_ARG, "ReadInputFile: unknown space geometry in " + k);
        }
        return PD_OK;
    };
    PDH_TRY(req("number_of_material_spaces"));
    int nms = 0;
    PDH_TRY(rd("number_of_material_spaces", 1, nms));
    _matSpaces.assign(std::max(nms, 0), Space());
    for (int i = 0; i < nms; ++i)
        PDH_TRY(read_space(keyword_append("material_space_", i + 1), true, nm, _matSpaces[i]));
    _delSpaces.clear();
    const bool hasDelKeyword = D.Find("number_of_deletion_spaces");
    if (hasDelKeyword) {
        int nd = 0;
        PDH_TRY(rd("number_of_deletion_spaces", 1, nd));
        _delSpaces.assign(std::max(nd, 0), Space());
        for (int i = 0; i < nd; ++i)
            PDH_TRY(read_space(keyword_append("deletion_space_", i + 1), false, 0, _delSpaces[i]));
    }
    PDH_TRY(req("number_of_boundary_spaces"));
    int nbs = 0;
    PDH_TRY(rd("number_of_boundary_spaces", 1, nbs));
    _bdrySpaces.assign(std::max(nbs, 0), Space());
    for (int i = 0; i < nbs; ++i)
        PDH_TRY(read_space(keyword_append("boundary_space_", i + 1), true, nb, _bdrySpaces[i]));
    // slits (keyword format of pdSlit.h:6-10)
    _slits.clear();
    if (D.Find("number_of_slits")) {
        int ns = 0;
        PDH_TRY(rd("number_of_slits", 1, ns));
        for (int i = 0; i < ns; ++i) {
            const std::string k = keyword_append("slit_", i + 1);
            int type = 0;
            PDH_TRY(rd(k, 1, type));
            if (type != 1) return Error(PD_ERR_ARG, "ReadInputFile: only rectangular slits (type 1) exist");
            for (int a = 0; a < 6; ++a) {
                double v = 0;
                PDH_TRY(rd(k, a + 2, v));
                _slits.push_back(v);
            }
        }
    }
    // control flags
    PDH_TRY(req("damping_coeff"));
    PDH_TRY(rd("damping_coeff", 1, _dampCoeff));
    PDH_TRY(req("bdryEff_on"));
    PDH_TRY(rd("bdryEff_on", 1, _bdryEffOn));
    _tolerance = 1.0e-4 * _gridSpacing;
    PDH_TRY(req("cci_on"));
    PDH_TRY(rd("cci_on", 1, _cciOn));
    if (_cciOn) {
        _fgiOn = _mlsOn = false;
        _intgPoint = 0;
        PDH_TRY(rd("cci_on", 2, _cciMdf));
    } else {
        PDH_TRY(req("fgi_on"));
        PDH_TRY(rd("fgi_on", 1, _fgiOn));
        _cciMdf = false;
        if (_fgiOn) {
            _intgPoint = 3;
            if (D.Find("intg_point")) PDH_TRY(rd("intg_point", 1, _intgPoint));
            _mlsOn = _intgPoint != 1;
            _rw = 3.0 * _gridSpacing;
            if (D.Find("support_domain_size")) PDH_TRY(rd("support_domain_size", 1, _rw));
            if (_intgPoint < 1 || _intgPoint > 8 || _intgPoint == 7)
                return Error(PD_ERR_ARG, "ReadInputFile: intg_point must be 1-6 or 8");
        } else {
            // adaptive trapezoid integration, pdDataManager.cpp:656-717
            PDH_TRY(req("ai_on"));
            PDH_TRY(rd("ai_on", 1, _aiOn));
            if (!_aiOn) return Error(PD_ERR_ARG, "ReadInputFile: no integration method is used! ");
            PDH_TRY(rd("ai_on", 2, _mlsOn));
            _rw = 3.0 * _gridSpacing;
            if (D.Find("support_domain_size")) PDH_TRY(rd("support_domain_size", 1, _rw));
            _intgPoint = 3;
            if (D.Find("intg_point")) PDH_TRY(rd("intg_point", 1, _intgPoint));
            _errorControlOn = false;
            _eps = 0.0;
            if (D.Find("error_control_on")) {
                PDH_TRY(rd("error_control_on", 1, _errorControlOn));
                if (_errorControlOn) {
                    _eps = 0.01;
                    if (D.Find("error_control_eps")) PDH_TRY(rd("error_control_eps", 1, _eps));
                }
            }
            if (_errorControlOn)
                return Error(PD_ERR_ARG, "ReadInputFile: error_control_on is not supported: the refinement reads MLS "
                                         "list entries the setup pass never filled (pdIntgManager2.cpp:174)");
            if (_intgPoint < 1 || _intgPoint > 3)
                return Error(PD_ERR_ARG, "ReadInputFile: the AI trapezoid index (intg_point) must be 1-3: above 3 "
                                         "the reference's rule refines a sum left by the previous integral");
        }
    }
#undef PDH_TRY
    const int n1 = (_cciOn || _aiOn) ? 1 : _intgPoint;
    _npt = n1 * n1 * n1;
    gauss_rule(n1, _abscis, _weights);
    EchoDeck(log, hasDelKeyword);
    _stage = true;
    return PD_OK;
}

namespace {

// pdBdryCondition::Print and the subclasses' type line (pdBdryCondition.cpp:
// 55-74, pdBdryConditionDispl.cpp:29-33, ...Veloc.cpp:20-24,
// ...DisplGrad.cpp:30-34, ...Tract.cpp:29-33)
void print_bc(std::ostream& os, int k, const BdryCondition& b) {
    os << "Boundary Condition " << k + 1 << "\n";
    os << "  Direction flag = " << b.dir[0] << "\t" << b.dir[1] << "\t" << b.dir[2] << "\n";
    os << "  Value = ";
    for (double v : b.value) os << v << "\t";
    os << "\n" << "  End time = " << b.end_time << "\t";
    os << (b.load_type == 1.0 ? "Loading type = Ramp loading" : "Loading type = Step loading") << "\n";
    switch (b.type) {
        case DISPL: os << "  Type: Prescribed Displacement\n"; break;
        case VELOC: os << "  Type: Prescribed Velocity\n"; break;
        case DISPLGRAD: os << "  Type: Prescribed Displacement Gradient \n"; break;
        default: os << "  Type: Traction Force\n"; break;
    }
}

// pdSpace::Print (pdSpace.cpp:87-100)
void print_space(std::ostream& os, int k, const Space& s) {
    os << "Space " << k + 1 << "\n";
    if (s.geo == 1)
        os << "  x1= " << s.lo[0] << "\t" << s.hi[0] << "\t" << " x2= " << s.lo[1] << "\t" << s.hi[1] << "\t"
           << " x3= " << s.lo[2] << "\t" << s.hi[2];
    else
        os << "  center= " << s.c1 << "\t" << s.c2 << "\t" << " radius= " << s.rad << "\t" << " x3= " << s.lo[2]
           << "\t" << s.hi[2];
}

}  // namespace

// The deck echo of ReadInputFile into pds_output.dat, line for line the
// reference's (pdDataManager.cpp:89-112,281-288,349-356,411-418,536-543,
// 733-753).
void pdDataManager::EchoDeck(std::ostream& log, bool deletion_keyword) const {
    log << "ReadInputFile: Problem title = " << _title << "\n"
        << "ReadInputFile: Grid center: x1 = " << _center[0] << ", x2 = " << _center[1] << ", x3 = " << _center[2]
        << "\n"
        << "ReadInputFile: Grid dimension = " << _dims[0] << " * " << _dims[1] << " * " << _dims[2] << "\n"
        << "ReadInputFile: Global grid spacing = " << _gridSpacing << "\n"
        << "ReadInputFile: Global grid horizon = " << _horizon << "\n"
        << "ReadInputFile: Total run time = " << _totalTime << "\n"
        << "ReadInputFile: Total run steps = " << _totalStep << "\n"
        << "ReadInputFile: Step dump frequency = " << _stepDumpFrequency << "\n";
    if (_fixedTimeStepOn) log << "ReadInputFile: Fixed time step = " << _fixedTimeStep << "\n";
    log << "\nReadInputFile: Total boundary condition number = " << _bcs.size() << "\n";
    for (size_t k = 0; k < _bcs.size(); ++k) {
        print_bc(log, (int)k, _bcs[k]);
        log << "\n";
    }
    log << "\nReadInputFile: Total material space number = " << _matSpaces.size() << "\n";
    for (size_t k = 0; k < _matSpaces.size(); ++k) {
        print_space(log, (int)k, _matSpaces[k]);
        log << "\n  Type: material space associates with material id = " << _matSpaces[k].ref << "\n\n";
    }
    if (deletion_keyword) {
        log << "\nReadInputFile: Total deletion space number = " << _delSpaces.size() << "\n";
        for (size_t k = 0; k < _delSpaces.size(); ++k) {
            print_space(log, (int)k, _delSpaces[k]);
            log << "\n";
        }
    }
    log << "\nReadInputFile: Total boundary space number = " << _bdrySpaces.size() << "\n";
    for (size_t k = 0; k < _bdrySpaces.size(); ++k) {
        print_space(log, (int)k, _bdrySpaces[k]);
        log << "\n  Type: boundary condition space associates with BC id = " << _bdrySpaces[k].ref << "\n\n";
    }
    log << "\nReadInputFile: Linear damping coefficient = " << _dampCoeff << "\n";
    log << "\nReadInputFile: Boundary effect compensation factor flag = " << _bdryEffOn << "\n";
    log << "\nReadInputFile: CCI integration method flag = " << _cciOn << "\n";
    if (_cciOn) log << "\nReadInputFile: Modified CCI beta flag = " << _cciMdf << "\n";
    log << "\nReadInputFile: Integration with fixed Gaussian points method flag = " << _fgiOn << "\n";
    if (_fgiOn) {
        log << "\nReadInputFile: Starting Gaussian points = " << _intgPoint << "\n";
        log << "\nReadInputFile: Moving least square flag = " << _mlsOn << "\n";
    }
    log << "\nReadInputFile: Adaptive integration method flag = " << _aiOn << "\n";
    if (_aiOn) {
        log << "\nReadInputFile: Moving least square flag = " << _mlsOn << "\n";
        log << "\nReadInputFile: Error control method flag = " << _errorControlOn << "\n";
        log << "\nReadInputFile: Error control accuracy = " << _eps << "\n";
        log << "\nReadInputFile: Starting trapezoidal index = " << _intgPoint << "\n";
    }
}

// pdDataManager::InitNode, pdDataManager.cpp:813-1098
int pdDataManager::InitNode() {
    if (!_stage) return Error(PD_ERR_ARG, "InitNode: ReadInputFile first");
    const double tol = _tolerance;
    _x.clear();
    for (int n = 1; n != _dims[2] + 1; ++n)
        for (int m = 1; m != _dims[1] + 1; ++m)
            for (int l = 1; l != _dims[0] + 1; ++l) {
                const double x1 = (l - (_dims[0] + 1) * 0.5) * _gridSpacing + _center[0];
                const double x2 = (m - (_dims[1] + 1) * 0.5) * _gridSpacing + _center[1];
                const double x3 = (n - (_dims[2] + 1) * 0.5) * _gridSpacing + _center[2];
                bool del = false;
                for (const Space& s : _delSpaces) del = del || s.Contains(x1, x2, x3, tol);
                if (!del) {
                    _x.push_back(x1);
                    _x.push_back(x2);
                    _x.push_back(x3);
                }
            }
    _numNodes = (int64_t)(_x.size() / 3);
    if (_numNodes > INT32_MAX) return Error(PD_ERR_ARG, "InitNode: too many nodes");
    _mat.assign(_numNodes, -1);
    _bc.assign(_numNodes, -1);
    for (int64_t i = 0; i < _numNodes; ++i) {
        const double* p = &_x[3 * i];
        // every material space overwrites: a node outside the last space
        // has no material (pdDataManager.cpp:937-955,960-970)
        for (const Space& s : _matSpaces) _mat[i] = s.Contains(p[0], p[1], p[2], tol) ? s.ref : -1;
        if (_mat[i] < 0) {
            std::ostringstream o;
            o << "InitNode: node " << i << " not in any material space!";
            return Error(PD_ERR_ARG, o.str());
        }
        for (const Space& s : _bdrySpaces)
            if (s.Contains(p[0], p[1], p[2], tol)) _bc[i] = s.ref;
    }
    _bdryEff.assign(_numNodes, 1.0);
    _nodesDone = true;
    std::ofstream log(_outFilePath.c_str(), std::ios::app);
    log << "\nInitNode: total node number = " << _numNodes << "\n"
        << "\nInitNode: Material association done \n"
        << "\nInitNode: boundary condition association done \n"
        << "\nInitNode: nodes initialization done \n";
    return PD_OK;
}

void pdDataManager::DeviceTables(std::vector<pd_material>& mats, std::vector<pd_bc>& bcs) const {
    mats.assign(_mats.size(), pd_material{});
    for (size_t k = 0; k < _mats.size(); ++k) {
        const Material& m = _mats[k];
        // spring constant as InitMaterial sets it (pdDataManager.cpp:1310-1322)
        mats[k].spring = m.type == 1 ? 18 * m.BulkModulus() / (kPI * std::pow(_horizon, 4.0)) : 0.0;
        mats[k].density = m.density;
        mats[k].ecrit = m.ecrit;
        for (int a = 0; a < 3; ++a) mats[k].grav[a] = m.grav[a];
    }
    bcs.assign(_bcs.size(), pd_bc{});
    for (size_t k = 0; k < _bcs.size(); ++k) {
        std::memset(&bcs[k], 0, sizeof(pd_bc));
        bcs[k].type = _bcs[k].type;
        for (int a = 0; a < 3; ++a) bcs[k].dir[a] = _bcs[k].dir[a];
        for (size_t a = 0; a < _bcs[k].value.size() && a < 9; ++a) bcs[k].value[a] = _bcs[k].value[a];
        bcs[k].end_time = _bcs[k].end_time;
        bcs[k].load_type = _bcs[k].load_type;
    }
}

int pdDataManager::EnsureContext() {
    if (_ctx) return PD_OK;
    if (!_nodesDone) return Error(PD_ERR_ARG, "EnsureContext: InitNode first");
    std::vector<pd_material> mats;
    std::vector<pd_bc> bcs;
    DeviceTables(mats, bcs);
    pd_problem P;
    std::memset(&P, 0, sizeof P);
    P.num_nodes = _numNodes;
    P.coords = _x.data();
    P.mat_id = _mat.data();
    P.bc_id = _bc.data();
    P.num_materials = (int32_t)mats.size();
    P.materials = mats.data();
    P.num_bcs = (int32_t)bcs.size();
    P.bcs = bcs.empty() ? nullptr : bcs.data();
    P.grid_spacing = _gridSpacing;
    P.horizon = _horizon;
    P.integration = _cciOn ? PD_INTG_CCI : (_aiOn ? PD_INTG_AI : PD_INTG_FGI);
    P.cci_modified = _cciMdf ? 1 : 0;
    P.intg_point = _cciOn ? 1 : _intgPoint;
    P.abscissae = _abscis.data();
    P.weights = _weights.data();
    P.damping = _dampCoeff;
    P.num_slits = (int32_t)(_slits.size() / 6);
    P.slits = _slits.empty() ? nullptr : _slits.data();
    P.spring_factor = _springFactor.empty() ? nullptr : _springFactor.data();
    int rc = pd_ctx_create(&P, &_ctx);
    if (rc != PD_OK) return Cuda(rc, "pd_ctx_create");
    pd_set_precision(_ctx, _precision);
    pd_set_energy(_ctx, _energy ? 1 : 0);
    // specimens that are complete boxes let the batch run the stencil force;
    // any other batch keeps the general kernels (the refusal changes nothing)
    if (_batch) pd_set_boxes(_ctx, (int)(_batchOffsets.size() - 1), _batchOffsets.data());
    _uploaded = false;
    return PD_OK;
}

// pdDataManager::InitBond, pdDataManager2.cpp:12-70, on the device
int pdDataManager::InitBond() {
    int rc = EnsureContext();
    if (rc != PD_OK) return rc;
    int64_t nh = 0, nb = 0;
    double mb = 0;
    if ((rc = pd_bond_search(_ctx, &nh, &nb, &mb)) != PD_OK) return Cuda(rc, "pd_bond_search");
    _famPtr.assign(_numNodes + 1, 0);
    _famCol.assign(std::max<int64_t>(nh, 0), 0);
    _famBroken.assign(std::max<int64_t>(nh, 0), 0);
    if ((rc = pd_get_family(_ctx, _famPtr.data(), _famCol.data(), _famBroken.data())) != PD_OK)
        return Cuda(rc, "pd_get_family");
    _numHalves = nh;
    _numBroken = nb;
    _minBondLength = mb;
    _bondsDone = true;
    _familyOnDevice = true;
    std::ofstream log(_outFilePath.c_str(), std::ios::app);
    log << "\nInitBond: total bonds number = " << nh / 2 << "\n"
        << "\nInitBond: bonds initialization done \n";
    return PD_OK;
}

int pdDataManager::SetFamily(const std::vector<int64_t>& row_ptr, const std::vector<int32_t>& col,
                             const std::vector<uint8_t>& broken, double min_bond) {
    if ((int64_t)row_ptr.size() != _numNodes + 1) return Error(PD_ERR_ARG, "SetFamily: row_ptr size");
    _famPtr = row_ptr;
    _famCol = col;
    _famBroken = broken.empty() ? std::vector<uint8_t>(col.size(), 0) : broken;
    _numHalves = (int64_t)col.size();
    _numBroken = 0;
    for (uint8_t b : _famBroken) _numBroken += b ? 1 : 0;
    _minBondLength = min_bond;
    _bondsDone = true;
    _uploaded = false;
    _familyOnDevice = false;
    if (_ctx) {
        int rc = pd_set_family(_ctx, _famPtr.data(), _famCol.data(), _famBroken.data());
        if (rc != PD_OK) return Cuda(rc, "pd_set_family");
        _familyOnDevice = true;
    }
    return PD_OK;
}

// pdDataManager::InitMaterial, pdDataManager.cpp:1297-1338
int pdDataManager::InitMaterial() {
    for (Material& m : _mats) m.spring = m.type == 1 ? 18 * m.BulkModulus() / (kPI * std::pow(_horizon, 4.0)) : 0.0;
    {
        // pdMaterial::Print and the type line (pdMaterial.cpp:100-106,
        // pdMaterialBond.cpp:15-19, pdMaterialState.cpp:16-20)
        std::ofstream log(_outFilePath.c_str(), std::ios::app);
        log << "\nInitMatieral: Total material number = " << _mats.size() << "\n";
        for (size_t k = 0; k < _mats.size(); ++k) {
            const Material& m = _mats[k];
            log << "Material " << k + 1 << "\n"
                << "  Young's modulus= " << m.ymod << "\t" << "Yield strength= " << m.sigmay << "\n"
                << "  Poisson's ratio= " << m.nu << "\t" << "Density= " << m.density << "\n"
                << "  Critical stretch= " << m.ecrit << "\t" << "Spring constant= " << m.spring << "\n"
                << (m.type == 1 ? "  Type: Bond-Based Material (PMB) \n" : "  Type: State-Based Material\n") << "\n";
        }
    }
    _minMaterialDensity = 1.0e10;
    _maxBulkSoundSpeed = 0.0;
    for (const Material& m : _mats) {
        _minMaterialDensity = std::min(_minMaterialDensity, m.density);
        _maxBulkSoundSpeed = std::max(_maxBulkSoundSpeed, m.BulkSoundSpeed());
    }
    _matDone = true;
    return PD_OK;
}

// pdDataManager::InitBdryEffectFactor, pdDataManager.cpp:1340-1473, with
// CalcBdryEffFactor / CalcBdryEffFactorTypeOne (pdDataManager2.cpp:1353-1485)
int pdDataManager::InitBdryEffectFactor() {
    if (!_bdryEffOn) return PD_OK;
    if (!_bondsDone || !_matDone) return Error(PD_ERR_ARG, "InitBdryEffectFactor: bonds and materials first");
    const double dx = _gridSpacing, delta = _horizon, tol = _tolerance;
    // full-sphere family count on a virtual lattice around the origin
    const int vd = 2 * (int(delta / dx) + 1);
    const double origin[3] = {0.0, 0.0, 0.0};
    int full = 0;
    for (int n = 1; n != vd + 1; ++n)
        for (int m = 1; m != vd + 1; ++m)
            for (int l = 1; l != vd + 1; ++l) {
                const double q[3] = {(l - vd * 0.5) * dx, (m - vd * 0.5) * dx, (n - vd * 0.5) * dx};
                double mn, mx;
                cube_distance(origin, q, dx, &mn, &mx);
                if (mn < delta + tol) ++full;
            }
    _numMaxFamily = full;
    const double lo[3] = {-_dims[0] * 0.5 * dx + _center[0], -_dims[1] * 0.5 * dx + _center[1],
                          -_dims[2] * 0.5 * dx + _center[2]};
    const double hi[3] = {_dims[0] * 0.5 * dx + _center[0], _dims[1] * 0.5 * dx + _center[1],
                          _dims[2] * 0.5 * dx + _center[2]};
    const double ns = (int(delta / dx)) * dx;
    const double vol = std::pow(dx, 3.0);
    auto type_one = [&](const Material& m, double h) {
        const double fullE = 3.0 * m.ymod;
        const double part = fullE - 0.5 * m.spring * kPI *
                                        (std::pow(delta, 4) / 4.0 - h * std::pow(delta, 3) / 3.0 + std::pow(h, 4) / 12.0);
        return fullE / part;
    };
    const bool cci_orig = _cciOn && !_cciMdf;
    for (int64_t i = 0; i < _numNodes; ++i) {
        const double a = _x[3 * i], b = _x[3 * i + 1], c = _x[3 * i + 2];
        const Material& m = _mats[_mat[i]];
        const int64_t nf = _famPtr[i + 1] - _famPtr[i];
        const bool in1 = b >= lo[1] + ns && b <= hi[1] - ns && c >= lo[2] + ns && c <= hi[2] - ns;
        const bool in2 = a >= lo[0] + ns && a <= hi[0] - ns && c >= lo[2] + ns && c <= hi[2] - ns;
        const bool in3 = a >= lo[0] + ns && a <= hi[0] - ns && b >= lo[1] + ns && b <= hi[1] - ns;
        double f;
        if (nf == full) f = 1.0;
        else if (a >= hi[0] - ns && a <= hi[0] && in1) f = type_one(m, hi[0] - a);
        else if (a >= lo[0] && a <= lo[0] + ns && in1) f = type_one(m, a - lo[0]);
        else if (b >= hi[1] - ns && b <= hi[1] && in2) f = type_one(m, hi[1] - b);
        else if (b >= lo[1] && b <= lo[1] + ns && in2) f = type_one(m, b - lo[1]);
        else if (c >= hi[2] - ns && c <= hi[2] && in3) f = type_one(m, hi[2] - c);
        else if (c >= lo[2] && c <= lo[2] + ns && in3) f = type_one(m, c - lo[2]);
        else {
            // energy ratio under a 1e-4 uniform dilatation
            const double e11 = 1.0e-4;
            const double eps[9] = {e11, 0.0, 0.0, 0.0, e11, 0.0, 0.0, 0.0, e11};
            double sum = 0.0;
            for (int64_t p = _famPtr[i]; p < _famPtr[i + 1]; ++p) {
                if (_famBroken[p]) continue;
                const double* Y = &_x[3 * (int64_t)_famCol[p]];
                const double x1 = Y[0] - a, x2 = Y[1] - b, x3 = Y[2] - c;
                const double e1 = eps[0] * x1 + eps[1] * x2 + eps[2] * x3;
                const double e2 = eps[3] * x1 + eps[4] * x2 + eps[5] * x3;
                const double e3 = eps[6] * x1 + eps[7] * x2 + eps[8] * x3;
                const double r = std::sqrt(x1 * x1 + x2 * x2 + x3 * x3);
                const double p1 = x1 + e1, p2 = x2 + e2, p3 = x3 + e3;
                const double pl = std::sqrt(p1 * p1 + p2 * p2 + p3 * p3);
                const double u = pl - r, s = u / r;
                const double el = (u <= 0 || (u > 0 && s <= m.ecrit)) ? 0.5 * (m.spring / r) * u * u : 0.0;
                const double beta = beta_factor(r, delta, dx, cci_orig);
                const double elj = el * beta * vol;
                sum += 0.5 * elj;
            }
            const double pinf = 3.0 * m.ymod * e11 * e11;
            f = pinf / sum;
        }
        _bdryEff[i] = f;
    }
    if (_ctx) {
        int rc = pd_set_bdry_eff(_ctx, _bdryEff.data());
        if (rc != PD_OK) return Cuda(rc, "pd_set_bdry_eff");
    }
    return PD_OK;
}

// pdDataManager::InitGridBoundary, pdDataManager.cpp:1100-1295: the model
// bounds are only used by output planes, which this build does not write.
int pdDataManager::InitGridBoundary() {
    // pdDataManager::InitGridBoundary, pdDataManager.cpp:1100-1170: the
    // lattice bounds, the force planes (total_force_plane, or the middle) and
    // the model space 50 spacings around; only the log uses them here
    double a[3], b[3], plane[3];
    for (int k = 0; k < 3; ++k) {
        a[k] = -(_dims[k] - 1) * 0.5 * _gridSpacing + _center[k];
        b[k] = (_dims[k] - 1) * 0.5 * _gridSpacing + _center[k];
        plane[k] = _forcePlaneOn ? _forcePlane[k] : 0.5 * (a[k] + b[k]);
    }
    const double deformed = 50.0 * _gridSpacing;
    std::ofstream log(_outFilePath.c_str(), std::ios::app);
    log << "\nInitGridBoundary: grid boundaries: x1a = " << a[0] << ", x1b = " << b[0] << "\n"
        << "InitGridBoundary: grid boundaries: x2a = " << a[1] << ", x2b = " << b[1] << "\n"
        << "InitGridBoundary: grid boundaries: x3a = " << a[2] << ", x3b = " << b[2] << "\n"
        << "\nInitGridBoundary: total force planes: x1= " << plane[0] << ", x2= " << plane[1] << ", x3= " << plane[2]
        << "\n"
        << "\nInitGridBoundary: model space boundaries: x1clo = " << a[0] - deformed << ", x1chi = " << b[0] + deformed
        << "\n"
        << "InitGridBoundary: model space boundaries: x2clo = " << a[1] - deformed << ", x2chi = " << b[1] + deformed
        << "\n"
        << "InitGridBoundary: model space boundaries: x3clo = " << a[2] - deformed << ", x3chi = " << b[2] + deformed
        << "\n";
    return PD_OK;
}

// pdDataManager::InitIntegrationPoint, pdDataManager2.cpp:106-309
int pdDataManager::InitIntegrationPoint() {
    const int rc = SetupIntegrationPoints();
    if (rc == PD_OK) {
        std::ofstream log(_outFilePath.c_str(), std::ios::app);
        log << "\nInitIntegrationPoint: integration points initialization done \n";
    }
    return rc;
}

// The adaptive-trapezoid form: the regions of every bond, and with MLS the
// contributors and the per-node coefficient lists of the trapezoid points
// (pdDataManager2.cpp:257-300), all on the host.
int pdDataManager::SetupAI() {
    if (!_bondsDone) return Error(PD_ERR_ARG, "InitIntegrationPoint: bonds first");
    const int64_t H = _famPtr.empty() ? 0 : _famPtr.back();
    int64_t R = 0;
    _aiRegPtr.assign(H + 1, 0);
    int rc = pd_ai_plan(_numNodes, _x.data(), _famPtr.data(), _famCol.data(), _gridSpacing, _horizon,
                        _aiRegPtr.data(), nullptr, 0, &R);
    if (rc != PD_OK) return Error(rc, "pd_ai_plan: bad family");
    _aiRegs.resize(std::max<int64_t>(R, 1));
    rc = pd_ai_plan(_numNodes, _x.data(), _famPtr.data(), _famCol.data(), _gridSpacing, _horizon, _aiRegPtr.data(),
                    _aiRegs.data(), R, &R);
    if (rc != PD_OK) return Error(rc, "pd_ai_plan");
    _aiTabPtr.clear();
    _aiTab.clear();
    if (_mlsOn) {
        mls_contributors(_numNodes, _x.data(), _famPtr.data(), _famCol.data(), _rw, _cbPtr, _cbIdx);
        _aiTabPtr.assign(_numNodes + 1, 0);
        int64_t nc = 0, bad = -1;
        rc = pd_ai_mls_table(_numNodes, _x.data(), _famPtr.data(), _famCol.data(), _aiRegPtr.data(), _aiRegs.data(),
                             _gridSpacing, _horizon, _intgPoint, _cbPtr.data(), _cbIdx.data(), _rw, _aiTabPtr.data(),
                             nullptr, 0, &nc, &bad);
        if (rc != PD_OK) return Error(rc, "pd_ai_mls_table");
        _aiTab.assign(std::max<int64_t>(nc, 1), 0.0);
        rc = pd_ai_mls_table(_numNodes, _x.data(), _famPtr.data(), _famCol.data(), _aiRegPtr.data(), _aiRegs.data(),
                             _gridSpacing, _horizon, _intgPoint, _cbPtr.data(), _cbIdx.data(), _rw, _aiTabPtr.data(),
                             _aiTab.data(), nc, &nc, &bad);
        if (rc == PD_ERR_SINGULAR) {
            std::ostringstream o;
            o << "pdMatrix::Gauss: Singular Matrix (MLS moment matrix of node " << bad << ")";
            return Error(rc, o.str());
        }
        if (rc != PD_OK) return Error(rc, "pd_ai_mls_table");
    }
    if (_ctx && _familyOnDevice) return UploadAI();
    return PD_OK;
}

int pdDataManager::UploadAI() {
    const bool m = _mlsOn;
    const int rc = pd_set_ai(_ctx, m ? 1 : 0, _aiRegPtr.data(), _aiRegs.data(), m ? _cbPtr.data() : nullptr,
                             m ? _cbIdx.data() : nullptr, m ? _aiTabPtr.data() : nullptr, m ? _aiTab.data() : nullptr);
    return rc == PD_OK ? PD_OK : Cuda(rc, "pd_set_ai");
}

int pdDataManager::SetupIntegrationPoints() {
    if (_aiOn) return SetupAI();
    if (!_mlsOn) return PD_OK;
    if (!_bondsDone) return Error(PD_ERR_ARG, "InitIntegrationPoint: bonds first");
    int64_t bad = -1;
    int rc = PD_OK;
    _mlsOnDevice = false;
    if (_deviceMls) {
        // the contributors and coefficients computed on the device; a batch
        // solves every specimen in its own frame, as BatchMLS does
        if ((rc = EnsureContext()) != PD_OK) return rc;
        if (!_familyOnDevice) {
            if ((rc = pd_set_family(_ctx, _famPtr.data(), _famCol.data(), _famBroken.data())) != PD_OK)
                return Cuda(rc, "pd_set_family");
            _familyOnDevice = true;
        }
        _cbPtr.clear();
        _cbIdx.clear();
        _coeff.clear();
        int64_t T = 0;
        rc = pd_mls_setup(_ctx, _rw, _batch ? _batchCoords.data() : nullptr, &T);
        if (rc != PD_OK) return Error(rc, std::string("pd_mls_setup: ") + pd_last_error());
        _mlsOnDevice = true;
        return PD_OK;
    }
    if (_batch) {
        rc = BatchMLS(&bad);
    } else {
        mls_contributors(_numNodes, _x.data(), _famPtr.data(), _famCol.data(), _rw, _cbPtr, _cbIdx);
        rc = mls_coefficients(_numNodes, _x.data(), _abscis.data(), _intgPoint, _gridSpacing, _cbPtr, _cbIdx, _rw,
                              _coeff, host_threads(), &bad);
    }
    if (rc == PD_ERR_ARG) return rc;
    if (rc != PD_OK) {
        std::ostringstream o;
        o << "pdMatrix::Gauss: Singular Matrix (MLS moment matrix of node " << bad << ")";
        return Error(rc, o.str());
    }
    if (_ctx) {
        rc = pd_set_mls(_ctx, _cbPtr.data(), _cbIdx.data(), _coeff.data());
        if (rc != PD_OK) return Cuda(rc, "pd_set_mls");
    }
    return PD_OK;
}

int64_t pdDataManager::NumContrib() const {
    if (_mlsOnDevice && _ctx) {
        int64_t T = 0;
        pd_mls_size(_ctx, &T);
        return T;
    }
    return _cbPtr.empty() ? 0 : _cbPtr.back();
}

int pdDataManager::FetchMLS() {
    if (!_mlsOnDevice || !_ctx || !_cbPtr.empty()) return PD_OK;
    int64_t T = 0;
    int rc = pd_mls_size(_ctx, &T);
    if (rc != PD_OK) return Cuda(rc, "pd_mls_size");
    _cbPtr.assign(_numNodes + 1, 0);
    _cbIdx.assign(T, 0);
    _coeff.assign((size_t)T * _npt, 0.0);
    rc = pd_get_mls(_ctx, _cbPtr.data(), _cbIdx.data(), _coeff.data());
    return rc == PD_OK ? PD_OK : Cuda(rc, "pd_get_mls");
}

int pdDataManager::UploadSetup() {
    int rc = EnsureContext();
    if (rc != PD_OK) return rc;
    if (_uploaded) return PD_OK;
    if (!_bondsDone) return Error(PD_ERR_ARG, "no family: InitBond first");
    if (!_familyOnDevice) {
        // the family was installed on the host (SetFamily) before the context existed
        rc = pd_set_family(_ctx, _famPtr.data(), _famCol.data(), _famBroken.data());
        if (rc != PD_OK) return Cuda(rc, "pd_set_family");
        _familyOnDevice = true;
    }
    if ((rc = pd_set_bdry_eff(_ctx, _bdryEff.data())) != PD_OK) return Cuda(rc, "pd_set_bdry_eff");
    if (_aiOn) {
        if (_aiRegPtr.empty()) return Error(PD_ERR_ARG, "no AI data: InitIntegrationPoint first");
        if ((rc = UploadAI()) != PD_OK) return rc;
    } else if (_mlsOn && !_mlsOnDevice) {
        if (_cbPtr.empty()) return Error(PD_ERR_ARG, "no MLS data: InitIntegrationPoint first");
        if ((rc = pd_set_mls(_ctx, _cbPtr.data(), _cbIdx.data(), _coeff.data())) != PD_OK) return Cuda(rc, "pd_set_mls");
    }
    _uploaded = true;
    return PD_OK;
}

int pdDataManager::SetPrecision(int p) {
    _precision = p;
    if (_ctx) return Cuda(pd_set_precision(_ctx, p), "pd_set_precision");
    return PD_OK;
}

int pdDataManager::SetEnergy(bool on) {
    _energy = on;
    if (_ctx) return Cuda(pd_set_energy(_ctx, on ? 1 : 0), "pd_set_energy");
    return PD_OK;
}

// pdDataManager::CalcStableTimeStep, pdDataManager2.cpp:6-10
double pdDataManager::CalcStableTimeStep() const {
    return _fixedTimeStepOn ? _fixedTimeStep : _safeFactor * _minBondLength / _maxBulkSoundSpeed;
}

int pdDataManager::InitDynamicSolve() {
    int rc = UploadSetup();
    if (rc != PD_OK) return rc;
    _kineticEnergyStep = _elasticEnergyStep = 0.0;
    return Cuda(pd_init_dynamic(_ctx), "pd_init_dynamic");
}

int pdDataManager::RK4(double dt, double time) {
    int rc = UploadSetup();
    if (rc != PD_OK) return rc;
    return Cuda(pd_rk4_step(_ctx, dt, time, &_kineticEnergyStep, &_elasticEnergyStep), "pd_rk4_step");
}

int pdDataManager::RK4Steps(double dt, double t0, int nsteps) {
    int rc = UploadSetup();
    if (rc != PD_OK) return rc;
    return Cuda(pd_rk4_steps(_ctx, dt, t0, nsteps), "pd_rk4_steps");
}

int pdDataManager::CalcBondBasedMotionRK4(double dt, double time, const std::vector<double>& us,
                                          std::vector<double>& k) {
    int rc = UploadSetup();
    if (rc != PD_OK) return rc;
    if ((int64_t)us.size() != 3 * _numNodes) return Error(PD_ERR_ARG, "CalcBondBasedMotionRK4: size");
    k.assign(3 * _numNodes, 0.0);
    return Cuda(pd_force_stage(_ctx, dt, time, us.data(), k.data()), "pd_force_stage");
}

int pdDataManager::CalcIntgPointDisplRK4(double time, const std::vector<double>& us) {
    int rc = UploadSetup();
    if (rc != PD_OK) return rc;
    if ((int64_t)us.size() != 3 * _numNodes) return Error(PD_ERR_ARG, "CalcIntgPointDisplRK4: size");
    return Cuda(pd_gather(_ctx, time, us.data()), "pd_gather");
}

int pdDataManager::StaticSolve(double time, int precision, double rtol, int maxit, std::vector<double>& u,
                               int* iters, double* relres) {
    int rc = UploadSetup();
    if (rc != PD_OK) return rc;
    if ((int64_t)u.size() != 3 * _numNodes) u.assign(3 * _numNodes, 0.0);
    return Cuda(pd_static_solve(_ctx, time, precision, rtol, maxit, u.data(), iters, relres), "pd_static_solve");
}

int pdDataManager::GetDispl(std::vector<double>& U) {
    U.assign(3 * _numNodes, 0.0);
    if (!_ctx) return PD_OK;
    return Cuda(pd_get_state(_ctx, U.data(), nullptr), "pd_get_state");
}

int pdDataManager::GetVeloc(std::vector<double>& V) {
    V.assign(3 * _numNodes, 0.0);
    if (!_ctx) return PD_OK;
    return Cuda(pd_get_state(_ctx, nullptr, V.data()), "pd_get_state");
}

int pdDataManager::SetState(const std::vector<double>& U, const std::vector<double>& V) {
    int rc = UploadSetup();
    if (rc != PD_OK) return rc;
    return Cuda(pd_set_state(_ctx, U.empty() ? nullptr : U.data(), V.empty() ? nullptr : V.data()), "pd_set_state");
}

// ------------------------------------------------------------------ pdSolve

int pdSolve::InitialProblem(pdDataManager& dat) {
    int rc;
    if ((rc = dat.ReadInputFile()) != PD_OK) return rc;
    if ((rc = dat.InitNode()) != PD_OK) return rc;
    if ((rc = dat.InitBond()) != PD_OK) return rc;
    if ((rc = dat.InitMaterial()) != PD_OK) return rc;
    if ((rc = dat.InitBdryEffectFactor()) != PD_OK) return rc;
    if ((rc = dat.InitGridBoundary()) != PD_OK) return rc;
    if ((rc = dat.InitIntegrationPoint()) != PD_OK) return rc;
    return PD_OK;
}

// DmgFrac of every node: pdNode::GetDmgFraction (pdNode.cpp:225-232), the
// int count of damaged bonds over the family size in int arithmetic.  Only
// the AI integrand counts (one per point past the critical stretch,
// pdIntgManager2.cpp:308); the Gauss-point and CCI paths leave it 0.
int pdDataManager::DamageFractions(std::vector<double>& f) {
    f.assign(_numNodes, 0.0);
    if (!_aiOn || !_ctx) return PD_OK;
    std::vector<int32_t> cnt(_numNodes, 0);
    const int rc = pd_get_damage(_ctx, nullptr, cnt.data());
    if (rc != PD_OK) return Cuda(rc, "pd_get_damage");
    for (int64_t i = 0; i < _numNodes; ++i) {
        const int nf = (int)(_famPtr[i + 1] - _famPtr[i]);
        f[i] = nf != 0 ? (double)(cnt[i] / nf) : 0.0;
    }
    return PD_OK;
}

// one node record as pdNode::Print writes it (pdNode.cpp:418-433)
static void print_node(std::ostream& os, int64_t i, const pdDataManager& dat, const std::vector<double>& U,
                       const std::vector<double>& V, const std::vector<double>& dmg) {
    const auto& x = dat.Coords();
    os << i << "\t" << x[3 * i] << "\t" << x[3 * i + 1] << "\t" << x[3 * i + 2] << "\t" << U[3 * i] << "\t"
       << U[3 * i + 1] << "\t" << U[3 * i + 2] << "\t" << V[3 * i] << "\t" << V[3 * i + 1] << "\t" << V[3 * i + 2]
       << "\t" << dat.MatIds()[i] << "\t" << dat.BcIds()[i] << "\t" << dat.BdryEff()[i] << "\t" << dmg[i];
}

int pdSolve::WriteTecplot(pdDataManager& dat, int step, double time) {
    std::vector<double> U, V, dmg;
    int rc;
    if ((rc = dat.GetDispl(U)) != PD_OK || (rc = dat.GetVeloc(V)) != PD_OK || (rc = dat.DamageFractions(dmg)) != PD_OK)
        return rc;
    std::ofstream out((dat.GetWkDir() + keyword_append("pds_tecplot_", step) + ".dat").c_str());
    out << "Tecplot formatting output mode\n";
    out.setf(std::ios::scientific);
    out.precision(5);
    out << "VARIABLES = \n ID X1 X2 X3 U1 U2 U3 V1 V2 V3 MatID BCID bdryEff DmgFrac \n"
        << "ZONE I=" << dat.GetGridDimension(0) << ", J=" << dat.GetGridDimension(1)
        << ", K=" << dat.GetGridDimension(2) << ", F=POINT\n\n";
    for (int64_t i = 0; i < dat.GetNumNode(); ++i) {
        print_node(out, i, dat, U, V, dmg);
        out << "\n";
    }
    (void)time;
    return PD_OK;
}

// ------------------------------------------------------------ PostAFD

namespace {

struct CoordKey {
    uint64_t a, b, c;
    bool operator==(const CoordKey& o) const { return a == o.a && b == o.b && c == o.c; }
};
struct CoordHash {
    size_t operator()(const CoordKey& k) const {
        return (size_t)((k.a * 0x9E3779B97F4A7C15ull) ^ (k.b * 0xC2B2AE3D27D4EB4Full) ^ (k.c * 0x165667B19E3779F9ull));
    }
};
CoordKey coord_key(double x1, double x2, double x3) {
    CoordKey k;
    std::memcpy(&k.a, &x1, 8);
    std::memcpy(&k.b, &x2, 8);
    std::memcpy(&k.c, &x3, 8);
    return k;
}

}  // namespace

int pdSolve::PostAFD(pdDataManager& dat, int step, const std::vector<AfdRequest>& requests) {
    int rc = dat.UploadSetup();
    if (rc != PD_OK) return rc;
    const int64_t N = dat.GetNumNode();
    const std::string in_path = dat.GetWkDir() + keyword_append("pds_tecplot_", step) + ".dat";
    std::ifstream in(in_path.c_str());
    if (!in) return dat.Error(PD_ERR_ARG, "ReadTecplotFile: pdMTEL tecplot output file not exist!");
    // the dump: four header lines, then one row per node
    // (pdDataManager3.cpp:1108-1130); displacements and boundary factors are
    // taken from it as written
    std::string line;
    for (int k = 0; k < 4; ++k) std::getline(in, line);
    std::vector<double> U(3 * (size_t)N, 0.0), bE(N, 1.0);
    for (int64_t k = 0; k < N; ++k) {
        int64_t id, mat, bc;
        double x1, x2, x3, u1, u2, u3, v1, v2, v3, be, dmg;
        if (!(in >> id >> x1 >> x2 >> x3 >> u1 >> u2 >> u3 >> v1 >> v2 >> v3 >> mat >> bc >> be >> dmg) || id < 0 ||
            id >= N)
            return dat.Error(PD_ERR_ARG, "PostAFD: " + in_path + " does not hold this model's nodes");
        U[3 * id] = u1;
        U[3 * id + 1] = u2;
        U[3 * id + 2] = u3;
        bE[id] = be;
    }
    const std::vector<double>& X = dat.Coords();
    std::unordered_map<CoordKey, int64_t, CoordHash> at;
    at.reserve((size_t)N * 2);
    for (int64_t i = 0; i < N; ++i) at.emplace(coord_key(X[3 * i], X[3 * i + 1], X[3 * i + 2]), i);
    const double h = dat.GetGridSpacing(), delta = dat.GetHorizon();
    const int ns = int(delta / h);
    const double ds = delta / ns;
    // items of one source: per direction the nodes at x_s - h (1 + is) e_d in
    // ascending id (the order CalcArealForceDensity lists them in,
    // pdDataManager3.cpp:463-480)
    auto sigma_of = [&](const std::vector<int64_t>& sources, std::vector<std::array<double, 9>>& sig) -> int {
        std::vector<int64_t> it_i, it_s;
        std::vector<int32_t> it_d;
        for (int64_t s : sources) {
            const double* xs = &X[3 * s];
            for (int d = 0; d < 3; ++d) {
                std::vector<int64_t> col;
                for (int is = 0; is != ns; ++is) {
                    double q[3] = {xs[0], xs[1], xs[2]};
                    q[d] = xs[d] - h * (1 + is);
                    auto f = at.find(coord_key(q[0], q[1], q[2]));
                    if (f != at.end()) col.push_back(f->second);
                }
                std::sort(col.begin(), col.end());
                for (int64_t i : col) {
                    it_i.push_back(i);
                    it_s.push_back(s);
                    it_d.push_back(d + 1);
                }
            }
        }
        std::vector<double> force(3 * it_i.size(), 0.0);
        const int r = pd_afd(dat.Context(), U.data(), bE.data(), (int64_t)it_i.size(), it_i.data(), it_s.data(),
                             it_d.data(), force.data());
        if (r != PD_OK) return dat.Cuda(r, "pd_afd");
        sig.assign(sources.size(), std::array<double, 9>{});
        size_t src = 0;
        for (size_t m = 0; m < it_i.size(); ++m) {
            while (it_s[m] != sources[src]) ++src;
            const int d = it_d[m] - 1;
            for (int a = 0; a < 3; ++a) sig[src][3 * d + a] += force[3 * m + a] * ds;
        }
        return PD_OK;
    };
    std::ofstream out((dat.GetWkDir() + keyword_append("pds_AFD_", step) + ".dat").c_str());
    for (const AfdRequest& q : requests) {
        std::vector<int64_t> src;
        if (q.kind == 1) {
            if (q.norm < 1 || q.norm > 3) return dat.Error(PD_ERR_ARG, "PostAFD: plane normal 1, 2 or 3");
            out << " norm = " << q.norm << ", location = " << q.coord << "\n";
            for (int64_t i = 0; i < N; ++i)
                if (X[3 * i + q.norm - 1] == q.coord) src.push_back(i);
        } else if (q.kind == 2) {
            if (q.node < 0 || q.node >= N) return dat.Error(PD_ERR_ARG, "PostAFD: node id out of range");
            src.push_back(q.node);
        } else {
            return dat.Error(PD_ERR_ARG, "PostAFD: request kind 1 (plane) or 2 (node)");
        }
        std::vector<std::array<double, 9>> sig;
        if ((rc = sigma_of(src, sig)) != PD_OK) return rc;
        for (size_t k = 0; k < src.size(); ++k) {
            const int64_t i = src[k];
            const double* x = &X[3 * i];
            const auto& g = sig[k];
            if (q.kind == 1) {
                out << i << "\t" << x[0] << "\t" << x[1] << "\t" << x[2];
                for (int a = 0; a < 9; ++a) out << "\t" << g[a];
                out << "\n";
            } else {
                out << " AFD at node " << x[0] << "\t" << x[1] << "\t" << x[2] << "\n";
                out << " sigma11 = " << g[0] << " sigma12 = " << g[1] << " sigma13 = " << g[2] << "\n"
                    << " sigma21 = " << g[3] << " sigma22 = " << g[4] << " sigma23 = " << g[5] << "\n"
                    << " sigma31 = " << g[6] << " sigma32 = " << g[7] << " sigma33 = " << g[8] << "\n\n";
            }
        }
    }
    return PD_OK;
}

// pdSolve::SolveDynamic, pdSolve.cpp:24-130
int pdSolve::SolveDynamic(pdDataManager& dat, bool write_files) {
    const int totalStep = dat.GetTotalStep();
    int lastStep = totalStep;
    const int dump = std::max(1, dat.GetStepDumpFrequency());
    const double totalTime = dat.GetTotalTime();
    const double stable = dat.CalcStableTimeStep();
    double t = 0.0, cur = stable;
    std::ofstream log, steps;
    if (write_files) {
        log.open((dat.GetWkDir() + "pds_output.dat").c_str(), std::ios::app);
        log.setf(std::ios::scientific);
        log.precision(5);
        log << "\n** Dynamic solution: starting from cycle 1 **\n";
        steps.open((dat.GetWkDir() + "pds_steps.dat").c_str());
        steps << "Data at given node for each time step output mode\n\n";
        steps << "Step Time ID X1 X2 X3 U1 U2 U3 V1 V2 V3 MatID BCID bdryEff DmgFrac \n";
        // the probe rows keep the stream's default format: the reference's
        // WriteEachStep (pdSolve.cpp:752-774) sets scientific notation on a
        // second stream but writes through the one SolveDynamic opened
    }
    int rc = dat.SetEnergy(write_files);
    if (rc != PD_OK) return rc;
    // probe node at (dx/2, dx/2, dx/2), pdSolve.cpp:764-771
    int64_t probe = -1;
    const double h = 0.5 * dat.GetGridSpacing();
    for (int64_t i = 0; i < dat.GetNumNode(); ++i)
        if (dat.Coords()[3 * i] == h && dat.Coords()[3 * i + 1] == h && dat.Coords()[3 * i + 2] == h) probe = i;
    for (int iter = 1; iter != totalStep + 1; ++iter) {
        t += cur;
        if (!(t <= totalTime)) break;
        if (write_files) {
            if ((rc = dat.InitDynamicSolve()) != PD_OK) return rc;
            if ((rc = dat.RK4(cur, t)) != PD_OK) return rc;
            log << iter << ": dt= " << cur << " t= " << t << " KE= " << dat.GetKinetTotal()
                << " EE= " << dat.GetElastStep() << "\n";
            if (iter == 1 || iter == lastStep || iter % dump == 0)
                if ((rc = WriteTecplot(dat, iter, t)) != PD_OK) return rc;
            if (probe >= 0) {
                std::vector<double> U, V, dmg;
                dat.GetDispl(U);
                dat.GetVeloc(V);
                if ((rc = dat.DamageFractions(dmg)) != PD_OK) return rc;
                steps << iter << "\t" << t << "\t";
                print_node(steps, probe, dat, U, V, dmg);
                steps << "\n";
            }
        } else {
            if ((rc = dat.RK4Steps(cur, t - cur, 1)) != PD_OK) return rc;
        }
        if (t + stable > totalTime && t != totalTime) {
            lastStep = iter + 1;
            cur = totalTime - t;
        }
    }
    if (!write_files && dat.Context()) pd_sync(dat.Context());
    return PD_OK;
}

// Static solve: the operator of pdSolve::AssembleEquation solved matrix-free
// (CG) at time = the stable time step of the first cycle (pdSolve.cpp:156-158).
int pdSolve::SolveStatic(pdDataManager& dat, int precision, double rtol, bool write_files) {
    std::vector<double> u(3 * (size_t)dat.GetNumNode(), 0.0);
    const double t = dat.CalcStableTimeStep();
    int iters = 0;
    double rel = 0.0;
    int rc = dat.StaticSolve(t, precision, rtol, 200000, u, &iters, &rel);
    if (rc != PD_OK) return rc;
    std::vector<double> V(u.size(), 0.0);
    if ((rc = dat.SetState(u, V)) != PD_OK) return rc;
    if (write_files) {
        std::ofstream log((dat.GetWkDir() + "pds_output.dat").c_str(), std::ios::app);
        log << "** Static solution: CG iterations = " << iters << ", relative residual = " << rel << " **\n";
        return WriteTecplot(dat, 1, t);
    }
    return PD_OK;
}

// ------------------------------------------------------------------ batch

int pdDataManager::InitBatch(const std::vector<pdDataManager*>& sp) {
    if (sp.empty()) return Error(PD_ERR_ARG, "InitBatch: no specimens");
    if (_ctx) return Error(PD_ERR_ARG, "InitBatch: this model already has a device context");
    for (size_t k = 0; k < sp.size(); ++k) {
        pdDataManager* m = sp[k];
        if (!m || !m->_stage) return Error(PD_ERR_ARG, "InitBatch: every specimen must have read its deck");
        int rc = PD_OK;
        if (!m->_nodesDone && (rc = m->InitNode()) != PD_OK) return Error(rc, "InitBatch: specimen: " + m->_err);
        if (!m->_matDone && (rc = m->InitMaterial()) != PD_OK) return Error(rc, "InitBatch: specimen: " + m->_err);
        const pdDataManager& f = *sp[0];
        if (m->_aiOn) return Error(PD_ERR_ARG, "InitBatch: the batching form runs the Gauss-point and CCI schemes");
        if (m->_gridSpacing != f._gridSpacing || m->_horizon != f._horizon || m->_cciOn != f._cciOn ||
            m->_cciMdf != f._cciMdf || m->_fgiOn != f._fgiOn || m->_mlsOn != f._mlsOn ||
            m->_intgPoint != f._intgPoint || m->_rw != f._rw || m->_dampCoeff != f._dampCoeff)
            return Error(PD_ERR_ARG, "InitBatch: specimens differ in spacing, horizon, integration or damping");
        if (m->_bdryEffOn) return Error(PD_ERR_ARG, "InitBatch: boundary effect factors are not batched");
        if (!m->_springFactor.empty() && (int64_t)m->_springFactor.size() != m->_numNodes)
            return Error(PD_ERR_ARG, "InitBatch: spring factor size");
    }
    const pdDataManager& f = *sp[0];
    _gridSpacing = f._gridSpacing;
    _horizon = f._horizon;
    _cciOn = f._cciOn;
    _cciMdf = f._cciMdf;
    _fgiOn = f._fgiOn;
    _mlsOn = f._mlsOn;
    _intgPoint = f._intgPoint;
    _npt = f._npt;
    _rw = f._rw;
    _dampCoeff = f._dampCoeff;
    _abscis = f._abscis;
    _weights = f._weights;
    _tolerance = f._tolerance;
    _totalStep = f._totalStep;
    _totalTime = f._totalTime;
    _fixedTimeStepOn = f._fixedTimeStepOn;
    _fixedTimeStep = f._fixedTimeStep;
    _safeFactor = f._safeFactor;
    _stepDumpFrequency = f._stepDumpFrequency;
    _bdryEffOn = false;
    _dims[0] = _dims[1] = _dims[2] = 0;
    _center[0] = _center[1] = _center[2] = 0.0;
    {
        std::ostringstream o;
        o << "batch of " << sp.size() << " specimens";
        _title = o.str();
    }
    // placement: shelves in the x-y plane, in lattice steps, with a gap
    // wider than the horizon plus a cell
    const double h = _gridSpacing;
    const int64_t gap = (int64_t)std::ceil(_horizon / h) + 3;
    const size_t K = sp.size();
    std::vector<std::array<double, 3>> lo(K);
    std::vector<std::array<int64_t, 3>> ext(K);
    double area = 0.0;
    int64_t widest = 0;
    for (size_t k = 0; k < K; ++k) {
        const pdDataManager& m = *sp[k];
        double l[3] = {1e300, 1e300, 1e300}, u[3] = {-1e300, -1e300, -1e300};
        for (int64_t i = 0; i < m._numNodes; ++i)
            for (int a = 0; a < 3; ++a) {
                l[a] = std::min(l[a], m._x[3 * i + a]);
                u[a] = std::max(u[a], m._x[3 * i + a]);
            }
        for (int a = 0; a < 3; ++a) {
            lo[k][a] = m._numNodes ? l[a] : 0.0;
            ext[k][a] = m._numNodes ? (int64_t)std::llround((u[a] - l[a]) / h) : 0;
        }
        area += (double)(ext[k][0] + gap) * (double)(ext[k][1] + gap);
        widest = std::max(widest, ext[k][0]);
    }
    const int64_t rowmax = std::max<int64_t>(widest, (int64_t)std::ceil(std::sqrt(area)));
    std::vector<std::array<int64_t, 3>> origin(K);
    int64_t cx = 0, cy = 0, rowh = 0;
    for (size_t k = 0; k < K; ++k) {
        if (cx > 0 && cx + ext[k][0] > rowmax) {
            cx = 0;
            cy += rowh + gap;
            rowh = 0;
        }
        origin[k] = {cx, cy, 0};
        cx += ext[k][0] + gap;
        rowh = std::max(rowh, ext[k][1]);
    }
    // merged node arrays
    _x.clear();
    _batchCoords.clear();
    _mat.clear();
    _bc.clear();
    _mats.clear();
    _bcs.clear();
    _slits.clear();
    _springFactor.clear();
    _batchOffsets.assign(1, 0);
    bool anyFactor = false;
    for (const pdDataManager* m : sp) anyFactor = anyFactor || !m->_springFactor.empty();
    // identical materials of different specimens become one entry, so that a
    // batch of one material runs the single-material kernels
    auto same = [](const Material& a, const Material& b) {
        return a.type == b.type && a.ymod == b.ymod && a.sigmay == b.sigmay && a.nu == b.nu &&
               a.ecrit == b.ecrit && a.density == b.density && a.grav[0] == b.grav[0] &&
               a.grav[1] == b.grav[1] && a.grav[2] == b.grav[2];
    };
    for (size_t k = 0; k < K; ++k) {
        const pdDataManager& m = *sp[k];
        const int bcBase = (int)_bcs.size();
        std::vector<int32_t> matMap(m._mats.size());
        for (size_t q = 0; q < m._mats.size(); ++q) {
            int found = -1;
            for (size_t e = 0; e < _mats.size() && found < 0; ++e)
                if (same(_mats[e], m._mats[q])) found = (int)e;
            if (found < 0) {
                found = (int)_mats.size();
                _mats.push_back(m._mats[q]);
            }
            matMap[q] = found;
        }
        double shift[3];
        for (int a = 0; a < 3; ++a) shift[a] = (double)origin[k][a] * h;
        for (int64_t i = 0; i < m._numNodes; ++i) {
            for (int a = 0; a < 3; ++a) {
                const double xa = m._x[3 * i + a];
                _x.push_back(shift[a] + (xa - lo[k][a]));
                _batchCoords.push_back(xa);
            }
            _mat.push_back(matMap[m._mat[i]]);
            _bc.push_back(m._bc[i] >= 0 ? m._bc[i] + bcBase : -1);
            if (anyFactor) _springFactor.push_back(m._springFactor.empty() ? 1.0 : m._springFactor[i]);
        }
        for (const BdryCondition& q : m._bcs) _bcs.push_back(q);
        for (size_t q = 0; q + 6 <= m._slits.size(); q += 6)
            for (int a = 0; a < 3; ++a)
                for (int e = 0; e < 2; ++e) _slits.push_back(shift[a] + (m._slits[q + 2 * a + e] - lo[k][a]));
        _batchOffsets.push_back(_batchOffsets.back() + m._numNodes);
    }
    _numNodes = _batchOffsets.back();
    if (_numNodes > INT32_MAX) return Error(PD_ERR_ARG, "InitBatch: too many nodes");
    _bdryEff.assign(_numNodes, 1.0);
    _batch = true;
    _stage = true;
    _nodesDone = true;
    _bondsDone = false;
    _uploaded = false;
    int rc = InitMaterial();
    if (rc != PD_OK) return rc;
    std::ofstream log(_outFilePath.c_str(), std::ios::app);
    log << "\nInitBatch: " << K << " specimens, total node number = " << _numNodes << "\n";
    return PD_OK;
}

// MLS of every specimen in its own coordinates, merged in node order
int pdDataManager::BatchMLS(int64_t* bad_node) {
    const size_t K = _batchOffsets.size() - 1;
    _cbPtr.assign(1, 0);
    _cbIdx.clear();
    _coeff.clear();
    for (size_t k = 0; k < K; ++k) {
        const int64_t o = _batchOffsets[k], n = _batchOffsets[k + 1] - o;
        std::vector<int64_t> fp(n + 1);
        std::vector<int32_t> fc;
        fc.reserve(_famPtr[o + n] - _famPtr[o]);
        for (int64_t i = 0; i <= n; ++i) fp[i] = _famPtr[o + i] - _famPtr[o];
        for (int64_t p = _famPtr[o]; p < _famPtr[o + n]; ++p) {
            const int64_t j = _famCol[p] - o;
            if (j < 0 || j >= n) return Error(PD_ERR_ARG, "InitIntegrationPoint: a bond joins two specimens");
            fc.push_back((int32_t)j);
        }
        std::vector<int64_t> cp;
        std::vector<int32_t> ci;
        std::vector<double> co;
        const double* xs = _batchCoords.data() + 3 * o;
        mls_contributors(n, xs, fp.data(), fc.data(), _rw, cp, ci);
        int64_t bad = -1;
        const int rc = mls_coefficients(n, xs, _abscis.data(), _intgPoint, _gridSpacing, cp, ci, _rw, co,
                                        host_threads(), &bad);
        if (rc != PD_OK) {
            *bad_node = bad >= 0 ? bad + o : -1;
            return rc;
        }
        const int64_t base = _cbPtr.back();
        for (int64_t i = 1; i <= n; ++i) _cbPtr.push_back(base + cp[i]);
        for (int32_t v : ci) _cbIdx.push_back((int32_t)(v + o));
        _coeff.insert(_coeff.end(), co.begin(), co.end());
    }
    return PD_OK;
}

}  // namespace pdh
