// Host side of the pdMTEL drop-in: the reference's pdDataManager / pdSolve
// API (pdDataManager.h:39-268, pdSolve.h:18-47) over the device C ABI.
//
// Differences from the reference, all on purpose:
//  * every method returns an int status (PD_OK or PD_ERR_*) instead of
//    calling exit(0) or throwing uncaught strings (pdDataManager.h:355-363);
//  * the working folder is given as an argument (SetWkDir), not read from
//    stdin, and decks with CR/LF line ends are accepted;
//  * the node/bond object graph is replaced by flat arrays: coordinates,
//    family CSR in ascending id order, MLS contributor CSR and coefficients,
//    which live on the GPU during the solve.
#pragma once

#include <cstdint>
#include <ostream>
#include <string>
#include <vector>

#include "pdmtel_b200.h"

namespace pdh {

// pdMaterial / pdMaterialBond (pdMaterial.h:13-64)
struct Material {
    int type = 1;          // 1 bond-based (PMB), 2 state-based (no force model)
    double ymod = 0, sigmay = 0, nu = 0.25, ecrit = 0, density = 0;
    double grav[3] = {0, 0, 0};
    double spring = 0;     // set by InitMaterial
    double BulkModulus() const { return ymod / (3.0 * (1.0 - 2.0 * nu)); }
    double BulkSoundSpeed() const;
};

// pdBdryCondition (pdBdryCondition.h:25-67)
struct BdryCondition {
    int type = 0;
    int dir[3] = {0, 0, 0};
    std::vector<double> value;
    double end_time = 0, load_type = 2;
};

// pdSpace and subclasses: cuboid (geo 1) or cylinder (geo 2)
struct Space {
    int geo = 1;
    int ref = -1;  // material or bc index
    double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    double rad = 0, c1 = 0, c2 = 0;
    bool Contains(double x1, double x2, double x3, double tol) const;
};

class pdDataManager {
public:
    pdDataManager();
    ~pdDataManager();
    pdDataManager(const pdDataManager&) = delete;
    pdDataManager& operator=(const pdDataManager&) = delete;

    // working folder holding pds_input.txt (replaces pdDataManager3.cpp:1503-1541)
    int SetWkDir(const std::string& dir);
    // output folder only (no deck): the log of a batch model
    int SetOutputDir(const std::string& dir);
    std::string GetWkDir() const { return _workDir; }

    // pdSolve::InitialProblem steps (pdSolve.cpp:10-22)
    int ReadInputFile();
    int InitNode();
    int InitBond();             // on the GPU (pd_bond_search)
    int InitMaterial();
    int InitBdryEffectFactor();
    int InitGridBoundary();
    int InitIntegrationPoint();
    // Batching (no counterpart in the reference): this model becomes one
    // problem over several specimens, each a model that has read its deck.
    // The specimens' nodes are placed side by side on one lattice with gaps
    // wider than the horizon, so InitBond finds no bond between specimens;
    // InitIntegrationPoint then solves each specimen's MLS in its own
    // coordinates.  Node ids run specimen by specimen (BatchOffsets).
    int InitBatch(const std::vector<pdDataManager*>& specimens);
    bool IsBatch() const { return _batch; }
    const std::vector<int64_t>& BatchOffsets() const { return _batchOffsets; }
    // installs a family computed elsewhere instead of InitBond (no GPU needed)
    int SetFamily(const std::vector<int64_t>& row_ptr, const std::vector<int32_t>& col,
                  const std::vector<uint8_t>& broken, double min_bond);

    // dynamic solve (pdDataManager.cpp:1767-2134, pdDataManager2.cpp:6-10,410-439)
    int InitDynamicSolve();
    double CalcStableTimeStep() const;
    int RK4(double dt, double time);
    int CalcBondBasedMotionRK4(double dt, double time, const std::vector<double>& displStep, std::vector<double>& k);
    int CalcIntgPointDisplRK4(double time, const std::vector<double>& displStep);
    int RK4Steps(double dt, double t0, int nsteps);  // device-resident stepping
    int SetPrecision(int precision);
    int SetEnergy(bool on);

    // static solve of the linearised operator (pdSolve.cpp:195-527)
    int StaticSolve(double time, int precision, double rtol, int maxit, std::vector<double>& u, int* iters,
                    double* relres);

    // state
    int DamageFractions(std::vector<double>& frac);  // DmgFrac of every node
    int GetDispl(std::vector<double>& U);
    int GetVeloc(std::vector<double>& V);
    int SetState(const std::vector<double>& U, const std::vector<double>& V);

    // getters (pdDataManager.h:107-158)
    int GetNumNode() const { return (int)_numNodes; }
    int64_t GetNumBond() const { return _numHalves / 2; }
    int64_t GetNumHalves() const { return _numHalves; }
    int64_t GetNumBroken() const { return _numBroken; }
    int GetTotalStep() const { return _totalStep; }
    int GetStepDumpFrequency() const { return _stepDumpFrequency; }
    double GetTotalTime() const { return _totalTime; }
    double GetGridSpacing() const { return _gridSpacing; }
    double GetHorizon() const { return _horizon; }
    double GetKinetTotal() const { return _kineticEnergyStep; }
    double GetElastStep() const { return _elasticEnergyStep; }
    int GetGridDimension(int a) const { return _dims[a]; }
    std::string GetProblemTitle() const { return _title; }
    int GetNumGaussPoints() const { return _npt; }
    int GetNumMaxFamily() const { return _numMaxFamily; }
    bool IsCCI() const { return _cciOn; }
    bool IsMLSOn() const { return _mlsOn; }
    double GetMinBondLength() const { return _minBondLength; }
    const std::string& LastError() const { return _err; }

    // flat data (host copies)
    const std::vector<double>& Coords() const { return _x; }
    const std::vector<int32_t>& MatIds() const { return _mat; }
    const std::vector<int32_t>& BcIds() const { return _bc; }
    const std::vector<int64_t>& FamilyPtr() const { return _famPtr; }
    const std::vector<int32_t>& FamilyCol() const { return _famCol; }
    const std::vector<uint8_t>& FamilyBroken() const { return _famBroken; }
    const std::vector<double>& BdryEff() const { return _bdryEff; }
    const std::vector<int64_t>& ContribPtr() const { return _cbPtr; }
    const std::vector<int32_t>& ContribIdx() const { return _cbIdx; }
    const std::vector<double>& Coeff() const { return _coeff; }
    // InitIntegrationPoint on the device (pd_mls_setup) instead of the host;
    // off by default: the host setup reproduces the reference bit for bit,
    // the device one up to the rounding of two powers (see pd_mls_setup)
    void SetDeviceSetup(bool on) { _deviceMls = on; }
    bool MLSOnDevice() const { return _mlsOnDevice; }
    int64_t NumContrib() const;
    // the MLS data of a device setup, copied to the host vectors above
    int FetchMLS();
    const std::vector<Material>& Materials() const { return _mats; }
    const std::vector<BdryCondition>& BCs() const { return _bcs; }
    pd_ctx* Context() { return _ctx; }
    int EnsureContext();
    // the material / BC tables as pd_ctx_create receives them
    void DeviceTables(std::vector<pd_material>& mats, std::vector<pd_bc>& bcs) const;
    const std::vector<double>& GaussAbscissae() const { return _abscis; }
    const std::vector<double>& GaussWeights() const { return _weights; }
    int GetIntgPoint() const { return _cciOn ? 1 : _intgPoint; }
    double GetDamping() const { return _dampCoeff; }
    void SetSpringFactor(const std::vector<double>& f) { _springFactor = f; }

private:
    friend class pdSolve;
    int Error(int code, const std::string& msg);
    int Cuda(int rc, const char* what);
    int UploadSetup();
    int BatchMLS(int64_t* bad_node);
    void EchoDeck(std::ostream& log, bool deletion_keyword) const;
    int SetupIntegrationPoints();
    int SetupAI();
    int UploadAI();

    std::string _workDir, _inFilePath, _outFilePath, _title, _err;
    std::vector<std::string> _deck;  // lines, trimmed
    int _dims[3] = {0, 0, 0};
    double _center[3] = {0, 0, 0};
    double _gridSpacing = 0, _horizon = 0, _totalTime = 0, _fixedTimeStep = 0, _safeFactor = 0.8;
    double _tolerance = 0, _dampCoeff = 0, _rw = 0;
    bool _forcePlaneOn = false;
    double _forcePlane[3] = {0, 0, 0};
    int _totalStep = 0, _stepDumpFrequency = 1, _intgPoint = 0, _npt = 1;
    bool _fixedTimeStepOn = false, _bdryEffOn = false, _cciOn = false, _cciMdf = false, _fgiOn = false,
         _mlsOn = false, _aiOn = false, _errorControlOn = false;
    double _eps = 0;
    // adaptive-trapezoid form: regions of every family entry, MLS tables
    std::vector<int64_t> _aiRegPtr, _aiTabPtr;
    std::vector<pd_ai_region> _aiRegs;
    std::vector<double> _aiTab;
    std::vector<Material> _mats;
    std::vector<BdryCondition> _bcs;
    std::vector<Space> _matSpaces, _delSpaces, _bdrySpaces;
    std::vector<double> _slits;  // [k][6]
    // nodes
    int64_t _numNodes = 0;
    std::vector<double> _x;      // [N][3]
    std::vector<int32_t> _mat, _bc;
    std::vector<double> _bdryEff;
    std::vector<double> _springFactor;
    // bonds
    std::vector<int64_t> _famPtr;
    std::vector<int32_t> _famCol;
    std::vector<uint8_t> _famBroken;
    int64_t _numHalves = 0, _numBroken = 0;
    double _minBondLength = 0;
    int _numMaxFamily = 0;
    // Gauss points / MLS
    std::vector<double> _abscis, _weights;
    std::vector<int64_t> _cbPtr;
    std::vector<int32_t> _cbIdx;
    std::vector<double> _coeff;
    // materials summary
    double _minMaterialDensity = 0, _maxBulkSoundSpeed = 0;
    // energies of the last step
    double _kineticEnergyStep = 0, _elasticEnergyStep = 0;
    // batch of specimens
    bool _batch = false;
    std::vector<int64_t> _batchOffsets;  // [specimens + 1]
    std::vector<double> _batchCoords;    // each specimen's own coordinates
    // device
    pd_ctx* _ctx = nullptr;
    bool _uploaded = false;
    bool _familyOnDevice = false;
    bool _deviceMls = false, _mlsOnDevice = false;
    int _precision = PD_PREC_FP64;
    bool _energy = true;
    bool _stage = false;  // ReadInputFile done
    bool _nodesDone = false, _bondsDone = false, _matDone = false;
};

// pdSolve (pdSolve.h:18-47)
class pdSolve {
public:
    static int InitialProblem(pdDataManager& dat);
    // the time loop of pdSolve.cpp:24-130 with the reference's output files
    // (pds_output.dat log, pds_steps.dat probe, pds_tecplot_<step>.dat)
    static int SolveDynamic(pdDataManager& dat, bool write_files = true);
    // matrix-free CG for the static operator; writes the displacement to the
    // node state and a Tecplot file
    static int SolveStatic(pdDataManager& dat, int precision = PD_PREC_FP64, double rtol = 1e-10,
                           bool write_files = true);
    static int WriteTecplot(pdDataManager& dat, int step, double time);
    // pdSolve::PostAFD (pdSolve.cpp:810-834, pdDataManager3.cpp:1101-1223)
    // without the console: reads pds_tecplot_<step>.dat and writes the areal
    // force density stress of every request to pds_AFD_<step>.dat.  A
    // request is a plane (kind 1: every node whose coordinate along `norm`
    // equals `coord`) or one node (kind 2: `node`).
    struct AfdRequest {
        int kind;
        int norm;
        double coord;
        int64_t node;
    };
    static int PostAFD(pdDataManager& dat, int step, const std::vector<AfdRequest>& requests);
};

// MLS/bdryEff/search helpers shared by the setup code (pd_setup.cpp)
int mls_contributors(int64_t n, const double* x, const int64_t* row_ptr, const int32_t* col, double rw,
                     std::vector<int64_t>& cb_ptr, std::vector<int32_t>& cb_idx);
int mls_coefficients(int64_t n, const double* x, const double* abscis, int n1, double dx,
                     const std::vector<int64_t>& cb_ptr, const std::vector<int32_t>& cb_idx, double rw,
                     std::vector<double>& coeff, int nthreads, int64_t* bad_node);
bool mls_point(const double* x, const int32_t* cb, int64_t nc, const double q[3], double rw, double* pw,
               double* out);
void gauss_rule(int n, std::vector<double>& abscis, std::vector<double>& weights);
void cube_distance(const double* pi, const double* pj, double dx, double* dmin, double* dmax);
double beta_factor(double dist, double delta, double dx, bool cci_original);

}  // namespace pdh
