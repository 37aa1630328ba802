// Test harness around the reference pdMTEL solver (built by oracle/build_ref.sh).
//
// This file is test infrastructure: it drives the reference's own public
// pdDataManager / pdSolve methods (pdSolve.cpp:10-22 InitialProblem,
// pdDataManager.cpp:1994-2134 RK4, pdDataManager.cpp:1767-1992
// CalcBondBasedMotionRK4, pdDataManager.cpp:2402-2495 CalcIntgPointDisplRK4)
// and dumps their FP64 state so that golden vectors can be generated and the
// reference CPU path can be timed.  Nothing in the product links it.
//
// The private members are opened only to set the working folder without the
// interactive SetWkDir() (pdDataManager3.cpp:1503-1541) and to read the
// per-node MLS data out.
//
// usage:
//   pdref_harness setup <dir> <out.bin>
//   pdref_harness force <dir> <out.bin> <t> <dt_stage>
//   pdref_harness traj  <dir> <out.bin> <nsteps> <dump_every>
//   pdref_harness time  <dir> <nsteps>
//   pdref_harness damp  <dir> <out.bin> <dt>
//   pdref_harness solve <dir>
//   pdref_harness afd   <dir> <script>
//
// solve: pdSolve::SolveDynamic (pdSolve.cpp:24-130) itself, which writes the
// reference's pds_output.dat log, pds_steps.dat probe and pds_tecplot_<step>
// files into <dir>.
//
// afd: pdSolve::PostAFD (pdSolve.cpp:810-834, pdDataManager3.cpp:442-635,
// 1101-1223), which asks the console for the Tecplot step to read and for the
// planes or nodes to evaluate; the answers come from the <script> file, and
// it writes pds_AFD_<step>.dat into <dir>.
//
// damp: the reference's matrix-free linearised stiffness pass,
// pdDataManager::CalcDampingCoeff (pdDataManager2.cpp:1616-1907), at three
// displacement fields: the per-dof sum of |K_ij| (absKVector, returned scaled
// by dt^2/4) and the damping coefficient 2 sqrt(u.Ku / u.Mu) of each field.
// These pin the static operator of pdSolve::AssembleEquation
// (pdSolve.cpp:195-527), whose coefficients are the same.
//
// <dir>/pds_input.txt is the deck.  An optional slit block
//   number_of_slits / k   and   slit_i / 1 x1lo x1hi x2lo x2hi x3lo x3hi
// marks every bond whose segment crosses the slit rectangle as broken right
// after InitBond, which is the deletion rule this project gives pdSlit
// (pdSlit.h:6-10 fixes only the keyword format).
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#define private public
#define protected public
#include "pdDataManager.h"
#include "pdSolve.h"
#include "pdVector.h"
#undef private
#undef protected

namespace {

struct Writer {
    FILE* f = nullptr;
    explicit Writer(const char* path) {
        f = std::fopen(path, "wb");
        if (!f) { std::perror(path); std::exit(3); }
        std::fwrite("PDB1", 1, 4, f);
    }
    ~Writer() { if (f) std::fclose(f); }
    void rec(const std::string& name, char type, const void* data, uint64_t count) {
        uint32_t nl = (uint32_t)name.size();
        std::fwrite(&nl, 4, 1, f);
        std::fwrite(name.data(), 1, nl, f);
        std::fwrite(&type, 1, 1, f);
        std::fwrite(&count, 8, 1, f);
        size_t es = type == 'd' ? 8 : type == 'q' ? 8 : 4;
        if (count) std::fwrite(data, es, count, f);
    }
    void d(const std::string& n, const std::vector<double>& v) { rec(n, 'd', v.data(), v.size()); }
    void i(const std::string& n, const std::vector<int32_t>& v) { rec(n, 'i', v.data(), v.size()); }
    void q(const std::string& n, const std::vector<int64_t>& v) { rec(n, 'q', v.data(), v.size()); }
    void d1(const std::string& n, double x) { rec(n, 'd', &x, 1); }
    void q1(const std::string& n, int64_t x) { rec(n, 'q', &x, 1); }
};

struct Slit { double lo[3], hi[3]; };

std::vector<std::string> deck_lines(const std::string& path) {
    std::ifstream in(path.c_str());
    std::vector<std::string> out;
    std::string line;
    while (std::getline(in, line)) {
        while (!line.empty() && (line.back() == ' ' || line.back() == '\r' || line.back() == '\t')) line.pop_back();
        size_t s = line.find_first_not_of(" \t");
        out.push_back(s == std::string::npos ? std::string() : line.substr(s));
    }
    return out;
}

std::vector<Slit> read_slits(const std::string& path) {
    std::vector<Slit> slits;
    std::vector<std::string> L = deck_lines(path);
    int n = 0;
    for (size_t k = 0; k + 1 < L.size(); ++k)
        if (L[k] == "number_of_slits") { std::istringstream(L[k + 1]) >> n; }
    for (int s = 1; s <= n; ++s) {
        std::string key = "slit_" + std::to_string(s);
        for (size_t k = 0; k + 1 < L.size(); ++k) {
            if (L[k] != key) continue;
            std::istringstream is(L[k + 1]);
            int type; Slit sl;
            is >> type >> sl.lo[0] >> sl.hi[0] >> sl.lo[1] >> sl.hi[1] >> sl.lo[2] >> sl.hi[2];
            slits.push_back(sl);
        }
    }
    return slits;
}

// Segment a->b crosses the axis-normal rectangle: the normal axis is the one
// with the smallest extent; a and b lie strictly on opposite sides of its
// plane and the crossing point lies inside the other two extents.
bool crosses(const Slit& s, const double a[3], const double b[3]) {
    int nrm = 0;
    double ext = s.hi[0] - s.lo[0];
    for (int k = 1; k < 3; ++k)
        if (s.hi[k] - s.lo[k] < ext) { ext = s.hi[k] - s.lo[k]; nrm = k; }
    double c = 0.5 * (s.lo[nrm] + s.hi[nrm]);
    double da = a[nrm] - c, db = b[nrm] - c;
    if (!((da < 0.0 && db > 0.0) || (da > 0.0 && db < 0.0))) return false;
    double t = (c - a[nrm]) / (b[nrm] - a[nrm]);
    for (int k = 0; k < 3; ++k) {
        if (k == nrm) continue;
        double p = a[k] + t * (b[k] - a[k]);
        if (p < s.lo[k] || p > s.hi[k]) return false;
    }
    return true;
}

void setup(pdDataManager& dat, const std::string& dir) {
    dat._myRank = 0;
    dat._numProcs = 1;
    dat._workDir = dir + "/";
    dat._inFilePath = dat._workDir + "pds_input.txt";
    dat._outFilePath = dat._workDir + "pds_output.dat";
    { std::ofstream o(dat._outFilePath.c_str()); }
    // pdSolve::InitialProblem (pdSolve.cpp:10-22) with the slit step inserted
    dat.ReadInputFile();
    dat.InitNode();
    dat.InitBond();
    std::vector<Slit> slits = read_slits(dat._inFilePath);
    for (pdBond* b : dat._bonds) {
        double a[3] = {b->GetNodeI()->GetX1(), b->GetNodeI()->GetX2(), b->GetNodeI()->GetX3()};
        double c[3] = {b->GetNodeJ()->GetX1(), b->GetNodeJ()->GetX2(), b->GetNodeJ()->GetX3()};
        for (const Slit& s : slits)
            if (crosses(s, a, c)) b->SetBreak(true);
    }
    dat.InitMaterial();
    dat.InitBdryEffectFactor();
    dat.InitGridBoundary();
    dat.InitIntegrationPoint();
}

int bc_index(pdDataManager& dat, pdBdryCondition* bc) {
    if (!bc) return -1;
    for (size_t k = 0; k < dat._BCs.size(); ++k)
        if (dat._BCs[k].GetPtr() == bc) return (int)k;
    return -2;
}

void dump_setup(pdDataManager& dat, Writer& w) {
    int N = dat.GetNumNode();
    std::vector<double> X(3 * (size_t)N), bE(N);
    std::vector<int32_t> mat(N), bc(N);
    std::vector<int64_t> fptr(N + 1, 0), cptr(N + 1, 0);
    std::vector<int32_t> fcol, broken, cidx;
    std::vector<double> coeff, gx;
    int G = 0;
    for (int i = 0; i < N; ++i) {
        pdNode* n = dat.GetNode(i);
        X[3 * i] = n->GetX1(); X[3 * i + 1] = n->GetX2(); X[3 * i + 2] = n->GetX3();
        bE[i] = n->GetBdryEffFactor();
        mat[i] = n->GetMaterial()->GetID();
        bc[i] = bc_index(dat, n->GetBC());
        for (int f = 0; f < n->GetNumFamily(); ++f) {
            fcol.push_back(n->GetFamilyNode(f)->GetID());
            broken.push_back(n->GetFamilyBond(f)->IsBreak() ? 1 : 0);
        }
        fptr[i + 1] = (int64_t)fcol.size();
        int ncb = n->GetContribNodeListSize();
        for (int k = 0; k < ncb; ++k) cidx.push_back(n->GetContribNode(k)->GetID());
        cptr[i + 1] = (int64_t)cidx.size();
        G = n->GetGaussianPointListSize();
        for (int g = 0; g < G; ++g) {
            pdGauss* gp = n->GetGaussianPoint(g);
            gx.push_back(gp->GetX1()); gx.push_back(gp->GetX2()); gx.push_back(gp->GetX3());
            if (dat._mlsOn) {
                pdVector* c = gp->GetCoeff();
                for (int k = 0; k < ncb; ++k) coeff.push_back(c->GetCoeff(k));
            }
        }
    }
    w.q1("n", N);
    w.d("coords", X);
    w.i("mat", mat);
    w.i("bc", bc);
    w.q("fam_ptr", fptr);
    w.i("fam_col", fcol);
    w.i("broken", broken);
    w.d("bdry_eff", bE);
    w.q("cb_ptr", cptr);
    w.i("cb_idx", cidx);
    w.q1("num_gauss", G);
    w.d("gauss_x", gx);
    w.d("coeff", coeff);
    w.d1("min_bond", dat._minBondLength);
    w.d1("dt", dat.CalcStableTimeStep());
    w.q1("num_bonds", dat.GetNumBond());
    std::vector<double> spring, ymod, dens, ecrit, grav;
    for (auto& m : dat._mats) {
        spring.push_back(m->GetSpringConstant());
        ymod.push_back(m->GetYoungModulus());
        dens.push_back(m->GetDensity());
        ecrit.push_back(m->GetCriticalStretch());
        grav.push_back(m->GetGrav1()); grav.push_back(m->GetGrav2()); grav.push_back(m->GetGrav3());
    }
    w.d("spring", spring);
    w.d("mat_ymod", ymod);
    w.d("mat_density", dens);
    w.d("mat_ecrit", ecrit);
    w.d("mat_grav", grav);
    std::vector<int32_t> bct, bcd;
    std::vector<double> bcv, bce, bcl;
    for (auto& h : dat._BCs) {
        pdBdryCondition* b = h.GetPtr();
        bct.push_back((int)b->GetType());
        bcd.push_back(b->GetDirFlagX1()); bcd.push_back(b->GetDirFlagX2()); bcd.push_back(b->GetDirFlagX3());
        for (int k = 0; k < 9; ++k) bcv.push_back(k < (int)b->_value.size() ? b->_value[k] : 0.0);
        bce.push_back(b->GetEndTime());
        bcl.push_back(b->_loadType);
    }
    w.i("bc_type", bct);
    w.i("bc_dir", bcd);
    w.d("bc_val", bcv);
    w.d("bc_end", bce);
    w.d("bc_load", bcl);
    std::vector<double> gw;
    if (N > 0)
        for (int g = 0; g < G; ++g) {
            pdGauss* gp = dat.GetNode(0)->GetGaussianPoint(g);
            gw.push_back(gp->GetWeightX1()); gw.push_back(gp->GetWeightX2()); gw.push_back(gp->GetWeightX3());
        }
    w.d("gw", gw);
    w.d("params", {dat._gridSpacing, dat._horizon, dat._dampCoeff, dat._rw, dat._gridCenterX1,
                   dat._gridCenterX2, dat._gridCenterX3, dat._totalTime});
    w.i("iparams", {(int)dat._cciOn, (int)dat._cciMdf, (int)dat._mlsOn, (int)dat._fgiOn, (int)dat._bdryEffOn,
                    dat._gridDimensionX1, dat._gridDimensionX2, dat._gridDimensionX3, dat._intgPoint,
                    dat._totalStep});
    if (dat._bdryEffOn) w.q1("num_max_family", dat._numMaxFamily);
}

// Deterministic, smooth-plus-wavy synthetic displacement and velocity fields.
void test_fields(pdDataManager& dat, std::vector<double>& u, std::vector<double>& v) {
    int N = dat.GetNumNode();
    double h = dat.GetGridSpacing();
    u.assign(3 * (size_t)N, 0.0);
    v.assign(3 * (size_t)N, 0.0);
    for (int i = 0; i < N; ++i) {
        pdNode* n = dat.GetNode(i);
        double x = n->GetX1() / h, y = n->GetX2() / h, z = n->GetX3() / h;
        u[3 * i + 0] = h * (1e-4 * (0.7 * x + 0.2 * y - 0.1 * z) + 2e-4 * std::sin(0.9 * x + 0.3 * y));
        u[3 * i + 1] = h * (1e-4 * (-0.3 * x + 0.5 * y + 0.25 * z) + 1e-4 * std::cos(0.4 * y - 0.8 * z));
        u[3 * i + 2] = h * (1e-4 * (0.1 * x - 0.2 * y + 0.6 * z) + 3e-4 * std::sin(0.5 * z + 0.7 * x));
        v[3 * i + 0] = 1e-3 * std::sin(0.2 * x + 0.1 * z);
        v[3 * i + 1] = 1e-3 * std::cos(0.3 * y);
        v[3 * i + 2] = -1e-3 * std::sin(0.25 * z - 0.15 * x);
    }
}

std::vector<double> node_state(pdDataManager& dat, int which) {
    int N = dat.GetNumNode();
    std::vector<double> out(3 * (size_t)N);
    for (int i = 0; i < N; ++i) {
        pdNode* n = dat.GetNode(i);
        if (which == 0) { out[3 * i] = n->GetU1(); out[3 * i + 1] = n->GetU2(); out[3 * i + 2] = n->GetU3(); }
        else if (which == 1) { out[3 * i] = n->GetV1(); out[3 * i + 1] = n->GetV2(); out[3 * i + 2] = n->GetV3(); }
        else { out[3 * i] = n->GetV1Buffer(); out[3 * i + 1] = n->GetV2Buffer(); out[3 * i + 2] = n->GetV3Buffer(); }
    }
    return out;
}

std::vector<double> gauss_u(pdDataManager& dat) {
    std::vector<double> out;
    for (int i = 0; i < dat.GetNumNode(); ++i) {
        pdNode* n = dat.GetNode(i);
        for (int g = 0; g < n->GetGaussianPointListSize(); ++g) {
            pdGauss* gp = n->GetGaussianPoint(g);
            out.push_back(gp->GetU1()); out.push_back(gp->GetU2()); out.push_back(gp->GetU3());
        }
    }
    return out;
}

int64_t evals_per_stage(pdDataManager& dat) {
    int64_t ev = 0;
    for (int i = 0; i < dat.GetNumNode(); ++i) {
        pdNode* n = dat.GetNode(i);
        for (int f = 0; f < n->GetNumFamily(); ++f) {
            if (n->GetFamilyBond(f)->IsBreak()) continue;
            ev += dat._cciOn ? 1 : n->GetFamilyNode(f)->GetGaussianPointListSize();
        }
    }
    return ev;
}

double now() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: %s setup|force|traj|time <dir> ...\n", argv[0]);
        return 2;
    }
    std::string mode = argv[1], dir = argv[2];
    pdDataManager dat;
    if (mode == "setup") {
        setup(dat, dir);
        Writer w(argv[3]);
        dump_setup(dat, w);
    } else if (mode == "force") {
        double t = std::atof(argv[4]), dts = std::atof(argv[5]);
        setup(dat, dir);
        Writer w(argv[3]);
        dump_setup(dat, w);
        std::vector<double> u, v;
        test_fields(dat, u, v);
        for (int i = 0; i < dat.GetNumNode(); ++i) {
            pdNode* n = dat.GetNode(i);
            n->SetU1(u[3 * i]); n->SetU2(u[3 * i + 1]); n->SetU3(u[3 * i + 2]);
            n->SetV1(v[3 * i]); n->SetV2(v[3 * i + 1]); n->SetV3(v[3 * i + 2]);
        }
        w.d("u_test", u);
        w.d("v_test", v);
        dat.InitDynamicSolve();
        dat.CalcIntgPointDisplRK4(t, u);
        w.d("ug", gauss_u(dat));
        std::vector<double> k;
        dat.CalcBondBasedMotionRK4(dts, t, u, k);
        w.d("k", k);
        w.d("vbuf", node_state(dat, 2));
        w.d("U_after", node_state(dat, 0));
        std::vector<double> eed;
        for (int i = 0; i < dat.GetNumNode(); ++i) eed.push_back(dat.GetNode(i)->GetElastEnergyDensity());
        w.d("eed", eed);
        // bonds broken by the stage (the AI integrand breaks them,
        // pdIntgManager2.cpp:301-308) and the per-node damaged-point counts
        std::vector<int32_t> broken_after, dmg;
        for (int i = 0; i < dat.GetNumNode(); ++i) {
            pdNode* n = dat.GetNode(i);
            for (int f = 0; f < n->GetNumFamily(); ++f) broken_after.push_back(n->GetFamilyBond(f)->IsBreak() ? 1 : 0);
            dmg.push_back(n->GetNumDmgBond());
        }
        w.i("broken_after", broken_after);
        w.i("dmg", dmg);
    } else if (mode == "traj") {
        int nsteps = std::atoi(argv[4]), every = std::atoi(argv[5]);
        setup(dat, dir);
        Writer w(argv[3]);
        dump_setup(dat, w);
        // the time loop of pdSolve::SolveDynamic (pdSolve.cpp:44-128) without file output
        double dt = dat.CalcStableTimeStep(), t = 0.0, total = dat.GetTotalTime();
        double cur = dt;
        int last = dat.GetTotalStep();
        std::vector<double> ke, ee, times;
        for (int it = 1; it <= nsteps && it <= dat.GetTotalStep(); ++it) {
            t += cur;
            if (!(t <= total)) break;
            dat.InitDynamicSolve();
            dat.RK4(cur, t);
            ke.push_back(dat.GetKinetTotal());
            ee.push_back(dat.GetElastStep());
            times.push_back(t);
            if (it % every == 0 || it == nsteps) {
                std::vector<int32_t> br;
                for (int i = 0; i < dat.GetNumNode(); ++i) {
                    pdNode* n = dat.GetNode(i);
                    for (int f = 0; f < n->GetNumFamily(); ++f) br.push_back(n->GetFamilyBond(f)->IsBreak() ? 1 : 0);
                }
                w.i("broken_" + std::to_string(it), br);
                w.d("U_" + std::to_string(it), node_state(dat, 0));
                w.d("V_" + std::to_string(it), node_state(dat, 1));
                w.d("ug_" + std::to_string(it), gauss_u(dat));
            }
            if (t + dt > total && t != total) { last = it + 1; cur = total - t; }
        }
        (void)last;
        w.d("ke", ke);
        w.d("ee", ee);
        w.d("times", times);
    } else if (mode == "damp") {
        double dt = std::atof(argv[4]);
        setup(dat, dir);
        Writer w(argv[3]);
        dump_setup(dat, w);
        const int N = dat.GetNumNode();
        std::vector<double> u, v;
        test_fields(dat, u, v);
        std::vector<double> damp;
        for (int f = 0; f < 3; ++f) {
            // field 0: the smooth test field; 1: the test velocity field used
            // as a displacement; 2: their sum with a node-wise alternating sign
            std::vector<double> uf(3 * (size_t)N);
            for (int i = 0; i < 3 * N; ++i)
                uf[i] = f == 0 ? u[i] : f == 1 ? 1e-3 * v[i] : u[i] + ((i / 3) % 2 ? -1e-3 : 1e-3) * v[i];
            for (int i = 0; i < N; ++i) {
                pdNode* n = dat.GetNode(i);
                n->SetU1(uf[3 * i]); n->SetU2(uf[3 * i + 1]); n->SetU3(uf[3 * i + 2]);
            }
            pdVector absK(3 * N);
            damp.push_back(dat.CalcDampingCoeff(dt, &absK));
            w.d("u_field_" + std::to_string(f), uf);
            if (f == 0) {
                std::vector<double> a(3 * (size_t)N);
                for (int i = 0; i < 3 * N; ++i) a[i] = absK.GetCoeff(i);
                w.d("absK", a);
            }
        }
        w.d("damp_coeff", damp);
        w.d1("damp_dt", dt);
    } else if (mode == "afd") {
        if (argc < 4) {
            std::fprintf(stderr, "afd needs a script file\n");
            return 2;
        }
        setup(dat, dir);
        std::ifstream script(argv[3]);
        std::streambuf* console = std::cin.rdbuf(script.rdbuf());
        pdSolve::PostAFD(dat);
        std::cin.rdbuf(console);
    } else if (mode == "solve") {
        setup(dat, dir);
        pdSolve::SolveDynamic(dat);
    } else if (mode == "time") {
        int nsteps = std::atoi(argv[3]);
        double t0 = now();
        setup(dat, dir);
        double t1 = now();
        double dt = dat.CalcStableTimeStep(), t = 0.0;
        std::vector<double> step_s;
        for (int it = 1; it <= nsteps; ++it) {
            t += dt;
            double a = now();
            dat.InitDynamicSolve();
            dat.RK4(dt, t);
            step_s.push_back(now() - a);
        }
        int64_t ev = evals_per_stage(dat);
        std::printf("{\"nodes\": %d, \"setup_s\": %.6f, \"evals_per_step\": %lld, \"step_s\": [",
                    dat.GetNumNode(), t1 - t0, (long long)(4 * ev));
        for (size_t k = 0; k < step_s.size(); ++k) std::printf("%s%.6f", k ? ", " : "", step_s[k]);
        std::printf("]}\n");
    } else {
        std::fprintf(stderr, "unknown mode %s\n", mode.c_str());
        return 2;
    }
    return 0;
}
