// Reference-oracle harness: drives ProteinDF's own DfCalcGridX, DfGenerateGrid
// and DfFunctional_* objects (compiled unmodified from the reference tree by
// oracle/ref/Makefile) on inputs written by the Python test tooling, and
// writes their outputs to a flat binary file.
//
// TEST INFRASTRUCTURE ONLY: this program is the checker that pins the CPU
// restatement (oracle/pdfxc_oracle.c) and the CUDA path, and the timed
// "reference" CPU baseline. Nothing in the product links or runs it.
//
// Modes
//   pdfxc_ref xc    <case.txt> <out.bin>   rho pass + Vxc pass of DfCalcGridX
//   pdfxc_ref grid  <case.txt> <out.bin>   atom-centred grid + Becke weights
//   pdfxc_ref func  <case.txt> <out.bin>   pointwise functional values
//   pdfxc_ref lebedev - <out.bin>          unit-sphere Lebedev tables
//   pdfxc_ref grad  <case.txt> <out.bin>   XC nuclear gradient + its SG-1 grid
//   pdfxc_ref density <case.txt> <out.bin> DfCalcGridX::gridDensity at listed points
//
// The XC mode follows DfCalcGridX::calcXCIntegForFockAndEnergy
// (src/libpdf/DfCalcGridX.cpp:2280-2315): calcRho_{LDA,GGA}_part (:1862-1962)
// on a grid matrix with xc-update = no, then buildVxc(gridMatrix, ...)
// (:2056-2193). The grid mode calls the same private members that
// DfGenerateGrid::generateGrid_atom (src/libpdf/DfGenerateGrid.cpp:934-1091)
// calls, shell by shell, so that single-centre and partition weights can be
// recorded separately.
#include <omp.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "DfCalcGridX.h"
#define private public
#define protected public
#include "DfGenerateGrid.h"
#undef private
#undef protected
#include "DfFunctional_B3LYP.h"
#include "DfFunctional_B88LYP.h"
#include "DfFunctional_Becke88.h"
#include "DfFunctional_HFS.h"
#include "DfFunctional_SVWN.h"
#include "TlLebedevGrid.h"
#include "TlPrdctbl.h"

namespace {

struct Case {
    std::map<std::string, std::string> kv;
    std::vector<std::string> atomSym;
    std::vector<double> atomCharge, atomXyz;
    // basis: element -> list of (shell, [(exp, coef)])
    std::map<std::string, std::vector<std::pair<char, std::vector<std::pair<double, double>>>>> basis;
    std::vector<std::string> basisOrder;

    std::string get(const std::string& k, const std::string& dflt = "") const {
        auto it = kv.find(k);
        return it == kv.end() ? dflt : it->second;
    }
};

Case readCase(const char* path) {
    Case c;
    std::ifstream in(path);
    if (!in) {
        std::fprintf(stderr, "cannot open %s\n", path);
        std::exit(2);
    }
    std::string line;
    while (std::getline(in, line)) {
        std::istringstream ss(line);
        std::string key;
        if (!(ss >> key) || key[0] == '#') continue;
        if (key == "atom") {
            std::string sym;
            double q, x, y, z;
            ss >> sym >> q >> x >> y >> z;
            c.atomSym.push_back(sym);
            c.atomCharge.push_back(q);
            c.atomXyz.insert(c.atomXyz.end(), {x, y, z});
        } else if (key == "cgto") {
            std::string el, shell;
            int nprim;
            ss >> el >> shell >> nprim;
            std::vector<std::pair<double, double>> prims(nprim);
            for (int i = 0; i < nprim; ++i) {
                std::getline(in, line);
                std::istringstream ps(line);
                ps >> prims[i].first >> prims[i].second;
            }
            if (!c.basis.count(el)) c.basisOrder.push_back(el);
            c.basis[el].push_back({shell[0], prims});
        } else {
            std::string rest;
            std::getline(ss, rest);
            const auto p = rest.find_first_not_of(' ');
            c.kv[key] = (p == std::string::npos) ? "" : rest.substr(p);
        }
    }
    return c;
}

TlSerializeData makeParam(const Case& c) {
    TlSerializeData p;
    p["method"] = "rks";
    p["guess"] = "core";
    p["K_engine"] = "conventional";
    p["XC_engine"] = "grid";
    p["xc_functional"] = c.get("functional", "SVWN");
    p["xc-update"] = "no";
    p["num_of_iterations"] = 1;
    p["num_of_atoms"] = (int)c.atomSym.size();
    p["xc-potential/grid-type"] = c.get("grid_type", "USER");
    p["grid/num_of_radial_shells"] = c.get("nrad", "75");
    p["grid/num_of_angular_points"] = c.get("nang", "302");
    p["grid/radial_quadorature_method"] = c.get("radial", "GC");
    p["grid/GC_mapping_type"] = c.get("gc_mapping", "TA");
    p["grid/partitioning_method"] = c.get("partition", "Becke");
    p["grid/pruning"] = c.get("pruning", "yes");
    TlSerializeData atoms;
    for (size_t i = 0; i < c.atomSym.size(); ++i) {
        TlSerializeData a;
        a["symbol"] = c.atomSym[i];
        a["label"] = "";
        a["charge"] = c.atomCharge[i];
        TlSerializeData xyz;
        for (int k = 0; k < 3; ++k) xyz.pushBack(c.atomXyz[3 * i + k]);
        a["xyz"] = xyz;
        atoms.pushBack(a);
    }
    p["coordinates"]["atoms"] = atoms;
    for (const auto& el : c.basisOrder) {
        TlSerializeData b;
        b["name"] = "basis-" + el;
        TlSerializeData cgtos;
        for (const auto& sh : c.basis.at(el)) {
            TlSerializeData cg;
            cg["scale_factor"] = 1.0;
            cg["shell_type"] = std::string(1, sh.first);
            TlSerializeData prims;
            for (const auto& pr : sh.second) {
                TlSerializeData pg;
                pg["exp"] = pr.first;
                pg["coef"] = pr.second;
                prims.pushBack(pg);
            }
            cg["pGTOs"] = prims;
            cgtos.pushBack(cg);
        }
        b["cGTOs"] = cgtos;
        p["basis_set"][el] = b;
        p["basis_set_j"][el] = b;  // only to satisfy auxiliary-basis lookups
        p["basis_set_xc"][el] = b;
    }
    return p;
}

std::vector<double> readDoubles(const std::string& path, size_t n) {
    std::vector<double> v(n);
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f || std::fread(v.data(), sizeof(double), n, f) != n) {
        std::fprintf(stderr, "cannot read %zu doubles from %s\n", n, path.c_str());
        std::exit(2);
    }
    std::fclose(f);
    return v;
}

// Output: records of [char name[32]][int64 n][n doubles].
struct Out {
    FILE* f;
    explicit Out(const char* path) : f(std::fopen(path, "wb")) {
        if (!f) {
            std::fprintf(stderr, "cannot write %s\n", path);
            std::exit(2);
        }
    }
    ~Out() { std::fclose(f); }
    void put(const char* name, const std::vector<double>& v) {
        char nm[32] = {0};
        std::strncpy(nm, name, 31);
        const long long n = (long long)v.size();
        std::fwrite(nm, 1, 32, f);
        std::fwrite(&n, sizeof(n), 1, f);
        std::fwrite(v.data(), sizeof(double), v.size(), f);
    }
    void put(const char* name, double x) { put(name, std::vector<double>(1, x)); }
};

bool isGGA(const std::string& fn) {
    return fn == "B3LYP" || fn == "BLYP" || fn == "B88LYP" || fn == "HFB";
}

DfFunctional_LDA* makeLDA(const std::string& fn) {
    if (fn == "SVWN") return new DfFunctional_SVWN();
    if (fn == "HFS") return new DfFunctional_HFS();
    std::fprintf(stderr, "unknown LDA functional %s\n", fn.c_str());
    std::exit(2);
}

DfFunctional_GGA* makeGGA(const std::string& fn) {
    if (fn == "B3LYP") return new DfFunctional_B3LYP();
    if (fn == "BLYP" || fn == "B88LYP") return new DfFunctional_B88LYP();
    if (fn == "HFB") return new DfFunctional_Becke88();
    std::fprintf(stderr, "unknown GGA functional %s\n", fn.c_str());
    std::exit(2);
}

class XcHarness : public DfCalcGridX {
   public:
    explicit XcHarness(TlSerializeData* p) : DfCalcGridX(p) {}
    const TlOrbitalInfo& orb() const { return this->m_tlOrbInfo; }
    int nao() const { return this->m_nNumOfAOs; }
    using DfCalcGridX::buildVxc;
    using DfCalcGridX::calcRho_GGA_part;
    using DfCalcGridX::calcRho_LDA_part;
    using DfCalcGridX::getAOs;
    using DfCalcGridX::getDAOs;
    using DfCalcGridX::getD2AOs;
    using DfCalcGridX::energyGradient_part;
};

class GridHarness : public DfGenerateGrid {
   public:
    explicit GridHarness(TlSerializeData* p) : DfGenerateGrid(p) {}
    using DfGenerateGrid::generateGrid_atom;
};

double seconds_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

int runXc(const Case& c, const char* outPath) {
    TlSerializeData param = makeParam(c);
    // DfObject reads num_of_AOs from the parameter set; build the AO table first.
    const TlOrbitalInfo orbProbe(param["coordinates"], param["basis_set"]);
    const int N = orbProbe.getNumOfOrbitals();
    param["num_of_AOs"] = N;
    XcHarness h(&param);

    const std::string fn = c.get("functional", "SVWN");
    const bool gga = isGGA(fn);
    // open shell: a second density (density_file_b) and the P_A, P_B overloads
    const bool uks = c.get("uks", "0") == "1";
    const long npts = std::atol(c.get("npts", "0").c_str());
    const int ncol = uks ? (gga ? 13 : 7) : (gga ? 9 : 6);
    const std::vector<double> grid = readDoubles(c.get("grid_file"), (size_t)npts * 5);
    const std::vector<double> P = readDoubles(c.get("density_file"), (size_t)N * N);
    const std::vector<double> Pb = uks ? readDoubles(c.get("density_file_b"), (size_t)N * N) : std::vector<double>();
    const int nthreads = std::atoi(c.get("threads", "1").c_str());
    omp_set_num_threads(nthreads > 0 ? nthreads : 1);

    TlDenseGeneralMatrix_Lapack gridMat(npts, ncol);
    for (long i = 0; i < npts; ++i)
        for (int k = 0; k < 5; ++k) gridMat.set(i, k, grid[5 * i + k]);
    TlDenseSymmetricMatrix_Lapack PA(N), PB(N);
    for (int i = 0; i < N; ++i)
        for (int j = 0; j <= i; ++j) {
            PA.set(i, j, P[(size_t)i * N + j]);
            if (uks) PB.set(i, j, Pb[(size_t)i * N + j]);
        }
    TlDenseSymmetricMatrix_Lapack F(N), FB(N);

    const auto t0 = std::chrono::steady_clock::now();
    if (gga) {
        uks ? h.calcRho_GGA_part(PA, PB, &gridMat) : h.calcRho_GGA_part(PA, &gridMat);
    } else {
        uks ? h.calcRho_LDA_part(PA, PB, &gridMat) : h.calcRho_LDA_part(PA, &gridMat);
    }
    const double tRho = seconds_since(t0);
    const auto t1 = std::chrono::steady_clock::now();
    double exc = 0.0;
    if (gga) {
        DfFunctional_GGA* f = makeGGA(fn);
        exc = uks ? h.buildVxc(gridMat, f, &F, &FB) : h.buildVxc(gridMat, f, &F);
        delete f;
    } else {
        DfFunctional_LDA* f = makeLDA(fn);
        exc = uks ? h.buildVxc(gridMat, f, &F, &FB) : h.buildVxc(gridMat, f, &F);
        delete f;
    }
    const double tVxc = seconds_since(t1);

    Out out(outPath);
    out.put("exc", exc);
    out.put("t_rho", tRho);
    out.put("t_vxc", tVxc);
    out.put("threads", (double)nthreads);
    std::vector<double> vxc((size_t)N * N), vxcb((size_t)N * N);
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) vxc[(size_t)i * N + j] = F.get(i, j), vxcb[(size_t)i * N + j] = FB.get(i, j);
    out.put("vxc", vxc);
    if (uks) out.put("vxc_b", vxcb);
    std::vector<double> rho((size_t)npts * (ncol - 5));
    double nel = 0.0, nelb = 0.0;
    const int colB = gga ? DfCalcGridX::GM_GGA_RHO_BETA : DfCalcGridX::GM_LDA_RHO_BETA;
    for (long i = 0; i < npts; ++i) {
        for (int k = 5; k < ncol; ++k) rho[(size_t)i * (ncol - 5) + (k - 5)] = gridMat.get(i, k);
        nel += gridMat.get(i, DfCalcGridX::GM_WEIGHT) * gridMat.get(i, 5);
        if (uks) nelb += gridMat.get(i, DfCalcGridX::GM_WEIGHT) * gridMat.get(i, colB);
    }
    out.put("rho", rho);
    out.put("nelec_alpha", nel);
    if (uks) out.put("nelec_beta", nelb);

    // AO table as the reference normalises and orders it (TlOrbitalInfoObject).
    const TlOrbitalInfo& orb = h.orb();
    std::vector<double> aoAtom(N), aoType(N), aoNprim(N), aoExp, aoCoef;
    for (int i = 0; i < N; ++i) {
        aoAtom[i] = orb.getAtomIndex(i);
        aoType[i] = orb.getBasisType(i);
        aoNprim[i] = orb.getCgtoContraction(i);
        for (int k = 0; k < orb.getCgtoContraction(i); ++k) {
            aoExp.push_back(orb.getExponent(i, k));
            aoCoef.push_back(orb.getCoefficient(i, k));
        }
    }
    out.put("ao_atom", aoAtom);
    out.put("ao_type", aoType);
    out.put("ao_nprim", aoNprim);
    out.put("ao_exp", aoExp);
    out.put("ao_coef", aoCoef);

    // AO values and gradients at the first few points (getAOs / getDAOs).
    const long ndump = std::min<long>(npts, std::atol(c.get("ao_dump", "0").c_str()));
    std::vector<double> phi, dphi;
    for (long i = 0; i < ndump; ++i) {
        const TlPosition r(grid[5 * i], grid[5 * i + 1], grid[5 * i + 2]);
        std::vector<double> a, dx, dy, dz;
        h.getAOs(r, &a);
        h.getDAOs(r, &dx, &dy, &dz);
        phi.insert(phi.end(), a.begin(), a.end());
        for (int k = 0; k < N; ++k) dphi.insert(dphi.end(), {dx[k], dy[k], dz[k]});
    }
    out.put("phi", phi);
    out.put("dphi", dphi);
    return 0;
}

int runGrid(const Case& c, const char* outPath) {
    TlSerializeData param = makeParam(c);
    GridHarness g(&param);
    const int natom = (int)c.atomSym.size();
    TlDenseGeneralMatrix_Lapack I3(3, 3);
    for (int k = 0; k < 3; ++k) I3.set(k, k, 1.0);

    std::vector<double> pts, wsingle, wfinal, atomIdx, radii;
    std::vector<double> finalGrid;  // x y z w atom, screened, per atom in order
    for (int a = 0; a < natom; ++a) {
        const int Z = TlPrdctbl::getAtomicNumber(c.atomSym[a]);
        const double rM = TlPrdctbl::getBraggSlaterRadii(Z);
        radii.push_back(rM);
        radii.push_back(g.getCovalentRadiiForBecke(Z));
        // a dummy atom has no grid of its own (generateGrid_atom skips atomic number 0)
        for (int i = 1; i <= g.nrgrid && Z != 0; ++i) {
            double ri = 0.0, wr = 0.0;
            if (g.radialGridType_ == DfGenerateGrid::RG_GaussChebyshev) {
                g.getRadialAbscissaAndWeight_GaussChebyshev(rM, g.nrgrid, i, &ri, &wr);
            } else {
                g.getRadialAbscissaAndWeight_EulerMaclaurin(rM, g.nrgrid, i, &ri, &wr);
            }
            if (ri > 30.0) continue;
            const int nang = g.getNumOfPrunedAnglarPoints(ri, g.nOgrid, Z);
            std::vector<TlPosition> sph(nang);
            std::vector<double> w(nang);
            g.getSphericalGrids(nang, ri, wr, g.coord_[a], I3, &sph, &w);
            std::vector<double> wp = w;
            if (g.partitioningMethod_ == DfGenerateGrid::Paritioning_Becke) {
                g.calcMultiCenterWeight_Becke(a, nang, sph, &wp);
            } else {
                g.calcMultiCenterWeight_SS(a, nang, sph, &wp);
            }
            for (int k = 0; k < nang; ++k) {
                pts.insert(pts.end(), {sph[k].x(), sph[k].y(), sph[k].z()});
                wsingle.push_back(w[k]);
                wfinal.push_back(wp[k]);
                atomIdx.push_back(a);
            }
        }
        std::vector<double> x, y, z, w;
        g.generateGrid_atom(I3, a, &x, &y, &z, &w);
        for (size_t k = 0; k < x.size(); ++k) finalGrid.insert(finalGrid.end(), {x[k], y[k], z[k], w[k], (double)a});
    }
    Out out(outPath);
    out.put("points", pts);
    out.put("w_single", wsingle);
    out.put("w_final", wfinal);
    out.put("atom", atomIdx);
    out.put("radii", radii);
    out.put("grid", finalGrid);
    return 0;
}

// XC nuclear gradient, DfCalcGridX::energyGradient (src/libpdf/DfCalcGridX.cpp:1073-1415):
// energyGradient_part over all atoms gives the AO-centre term Fxc_f (then x2 for
// RKS, as energyGradient does) and the grid-weight term Fxc_w separately. The
// grid is the one energyGradient_part builds itself, DfGenerateGrid::getGrids
// (SG-1, src/libpdf/DfGenerateGrid.cpp:2091-2257), recorded here atom by atom
// so that other engines can be run on the same points.
int runGrad(const Case& c, const char* outPath) {
    TlSerializeData param = makeParam(c);
    const TlOrbitalInfo orbProbe(param["coordinates"], param["basis_set"]);
    const int N = orbProbe.getNumOfOrbitals();
    param["num_of_AOs"] = N;
    XcHarness h(&param);
    const int natom = (int)c.atomSym.size();
    const std::string fn = c.get("functional", "SVWN");
    const std::vector<double> P = readDoubles(c.get("density_file"), (size_t)N * N);
    TlDenseSymmetricMatrix_Lapack PA(N);
    for (int i = 0; i < N; ++i)
        for (int j = 0; j <= i; ++j) PA.set(i, j, P[(size_t)i * N + j]);

    TlDenseGeneralMatrix_Lapack Ff(natom, 3), Fw(natom, 3);
    const auto t0 = std::chrono::steady_clock::now();
    double exc = 0.0;
    if (isGGA(fn)) {
        DfFunctional_GGA* f = makeGGA(fn);
        exc = h.energyGradient_part(PA, f, 0, natom, &Ff, &Fw);
        delete f;
    } else {
        DfFunctional_LDA* f = makeLDA(fn);
        exc = h.energyGradient_part(PA, f, 0, natom, &Ff, &Fw);
        delete f;
    }
    const double tGrad = seconds_since(t0);
    Ff *= 2.0;  // rks, as energyGradient does

    DfGenerateGrid g(&param);
    std::vector<double> pts, wsingle, wpart, atomIdx;
    for (int a = 0; a < natom; ++a) {
        std::vector<TlPosition> grids;
        std::vector<double> ws, wp;
        g.getGrids(a, &grids, &ws, &wp);
        for (size_t k = 0; k < grids.size(); ++k) {
            pts.insert(pts.end(), {grids[k].x(), grids[k].y(), grids[k].z()});
            wsingle.push_back(ws[k]);
            wpart.push_back(wp[k]);
            atomIdx.push_back(a);
        }
    }
    Out out(outPath);
    std::vector<double> ff(3 * (size_t)natom), fw(3 * (size_t)natom);
    for (int a = 0; a < natom; ++a)
        for (int k = 0; k < 3; ++k) ff[3 * a + k] = Ff.get(a, k), fw[3 * a + k] = Fw.get(a, k);
    out.put("grad_orbital", ff);
    out.put("grad_weight", fw);
    out.put("exc", exc);
    out.put("t_grad", tGrad);
    out.put("points", pts);
    out.put("w_single", wsingle);
    out.put("w_partition", wpart);
    out.put("atom", atomIdx);
    return 0;
}

// Pointwise functional values through the overloads buildVxc uses
// (RKS: src/libpdf/DfCalcGridX.cpp:2076-2087, :2164-2185) and the
// open-shell ones the reference unit tests use.
int runFunc(const Case& c, const char* outPath) {
    const std::string fn = c.get("functional", "SVWN");
    const long n = std::atol(c.get("npts", "0").c_str());
    const std::vector<double> in = readDoubles(c.get("input_file"), (size_t)n * 5);
    std::vector<double> res;  // per point: f, vrhoA, vrhoB, vgaa, vgab, vgbb, f_rks, vr_rks, vgaa_rks, vgab_rks
    for (long i = 0; i < n; ++i) {
        const double ra = in[5 * i], rb = in[5 * i + 1], gaa = in[5 * i + 2], gab = in[5 * i + 3], gbb = in[5 * i + 4];
        double v[10] = {0};
        if (isGGA(fn)) {
            DfFunctional_GGA* f = makeGGA(fn);
            v[0] = f->getFunctional(ra, rb, gaa, gab, gbb);
            f->getDerivativeFunctional(ra, rb, gaa, gab, gbb, &v[1], &v[2], &v[3], &v[4], &v[5]);
            v[6] = f->getFunctional(ra, gaa);
            f->getDerivativeFunctional(ra, gaa, &v[7], &v[8], &v[9]);
            delete f;
        } else {
            DfFunctional_LDA* f = makeLDA(fn);
            v[0] = f->getFunctional(ra, rb);
            f->getDerivativeFunctional(ra, rb, &v[1], &v[2]);
            v[6] = f->getFunctional(ra, ra);
            f->getDerivativeFunctional(ra, &v[7]);
            delete f;
        }
        res.insert(res.end(), v, v + 10);
    }
    Out out(outPath);
    out.put("values", res);
    return 0;
}

// Unit-sphere Lebedev tables for every order the reference supports
// (src/libpdftl/TlLebedevGrid.cpp), as used by getSphericalGrids.
// rho(r) = phi(r)^T P phi(r) at the points of points_file (npts x 3) through the
// reference's DfCalcGridX::gridDensity (src/libpdf/DfCalcGridX.cpp:1038-1044), one
// call per point as TlDensField::makeDensFld makes them (src/tools/TlDensField.cpp:35-53).
std::vector<double> referenceDensities(TlSerializeData* param, const TlDenseSymmetricMatrix_Lapack& P,
                                       const std::vector<double>& xyz) {
    DfCalcGridX e(param);
    std::vector<double> rho(xyz.size() / 3, 0.0);
    for (size_t k = 0; k < rho.size(); ++k) e.gridDensity(P, TlPosition(xyz[3 * k], xyz[3 * k + 1], xyz[3 * k + 2]), &rho[k]);
    return rho;
}

TlDenseSymmetricMatrix_Lapack readSymmetric(const Case& c, int N) {
    const std::vector<double> P = readDoubles(c.get("density_file"), (size_t)N * N);
    TlDenseSymmetricMatrix_Lapack PA(N);
    for (int i = 0; i < N; ++i)
        for (int j = 0; j <= i; ++j) PA.set(i, j, P[(size_t)i * N + j]);
    return PA;
}

int runDensity(const Case& c, const char* outPath) {
    TlSerializeData param = makeParam(c);
    const TlOrbitalInfo orbProbe(param["coordinates"], param["basis_set"]);
    const int N = orbProbe.getNumOfOrbitals();
    param["num_of_AOs"] = N;
    const int npts = std::atoi(c.get("npts").c_str());
    const std::vector<double> xyz = readDoubles(c.get("points_file"), (size_t)npts * 3);
    Out out(outPath);
    out.put("rho", referenceDensities(&param, readSymmetric(c, N), xyz));
    return 0;
}

int runLebedev(const char* outPath) {
    TlLebedevGrid leb;
    const std::vector<int> orders = leb.getSupportedGridNumber();
    Out out(outPath);
    out.put("orders", std::vector<double>(orders.begin(), orders.end()));
    for (int n : orders) {
        std::vector<TlPosition> pts;
        std::vector<double> w;
        leb.getGrids(n, &pts, &w);
        std::vector<double> v;
        for (int k = 0; k < n; ++k) v.insert(v.end(), {pts[k].x(), pts[k].y(), pts[k].z(), w[k]});
        char name[32];
        std::snprintf(name, sizeof(name), "leb_%d", n);
        out.put(name, v);
    }
    return 0;
}

#ifdef PDFXC_DROPIN
// Drop-in check (built as oracle/_ref/pdfxc_dropin, linked with libpdfxc):
// the reference DfCalcGridX and DfCalcGridX_B200 on the same parameter set,
// grid-matrix file and density, through the reference's own matrix classes,
// for two SCF iterations (the second with xc-update on P_A/2, so the stored
// rho columns of the first are read back from the grid-matrix file).
}  // namespace
#include "DfCalcGridX_B200.h"
#include "DfGenerateGrid_B200.h"
namespace {

class GridFileWriter : public DfObject {
   public:
    explicit GridFileWriter(TlSerializeData* p) : DfObject(p) {}
    void save(int iteration, const TlDenseGeneralMatrix_Lapack& g) { this->saveGridMatrix(iteration, g); }
};

template <class Engine, class Functional>
double runEngine(TlSerializeData& param, int iteration, const TlDenseSymmetricMatrix_Lapack& P,
                 Functional* f, TlDenseSymmetricMatrix_Lapack* F) {
    param["num_of_iterations"] = iteration;
    Engine e(&param);
    return e.calcXCIntegForFockAndEnergy(P, f, F);
}

int runDropin(const Case& c, const char* outPath) {
    TlSerializeData param = makeParam(c);
    const TlOrbitalInfo orbProbe(param["coordinates"], param["basis_set"]);
    const int N = orbProbe.getNumOfOrbitals();
    param["num_of_AOs"] = N;
    param["xc-update"] = "yes";
    param["control"]["file_base_name"]["grid_matrix"] = "grid_%s.mat";
    const std::string fn = c.get("functional", "SVWN");
    const bool gga = isGGA(fn);
    const long npts = std::atol(c.get("npts", "0").c_str());
    const int ncol = gga ? 9 : 6;
    const std::vector<double> grid = readDoubles(c.get("grid_file"), (size_t)npts * 5);
    const std::vector<double> P = readDoubles(c.get("density_file"), (size_t)N * N);
    TlDenseGeneralMatrix_Lapack gridMat(npts, ncol);
    for (long i = 0; i < npts; ++i)
        for (int k = 0; k < 5; ++k) gridMat.set(i, k, grid[5 * i + k]);
    TlDenseSymmetricMatrix_Lapack PA(N), PA2(N);
    for (int i = 0; i < N; ++i)
        for (int j = 0; j <= i; ++j) PA.set(i, j, P[(size_t)i * N + j]), PA2.set(i, j, 0.5 * P[(size_t)i * N + j]);
    Out out(outPath);
    for (int engine = 0; engine < 2; ++engine) {
        GridFileWriter(&param).save(0, gridMat);
        double e1 = 0, e2 = 0;
        TlDenseSymmetricMatrix_Lapack F1(N), F2(N);
        // iteration 1 with P_A/2, iteration 2 with the difference P_A/2 (xc-update)
        if (gga) {
            DfFunctional_GGA* f = makeGGA(fn);
            e1 = engine ? runEngine<DfCalcGridX_B200>(param, 1, PA2, f, &F1) : runEngine<DfCalcGridX>(param, 1, PA2, f, &F1);
            e2 = engine ? runEngine<DfCalcGridX_B200>(param, 2, PA2, f, &F2) : runEngine<DfCalcGridX>(param, 2, PA2, f, &F2);
            delete f;
        } else {
            DfFunctional_LDA* f = makeLDA(fn);
            e1 = engine ? runEngine<DfCalcGridX_B200>(param, 1, PA2, f, &F1) : runEngine<DfCalcGridX>(param, 1, PA2, f, &F1);
            e2 = engine ? runEngine<DfCalcGridX_B200>(param, 2, PA2, f, &F2) : runEngine<DfCalcGridX>(param, 2, PA2, f, &F2);
            delete f;
        }
        std::vector<double> v1((size_t)N * N), v2((size_t)N * N);
        for (int i = 0; i < N; ++i)
            for (int j = 0; j < N; ++j) v1[(size_t)i * N + j] = F1.get(i, j), v2[(size_t)i * N + j] = F2.get(i, j);
        const char* tag = engine ? "b200" : "ref";
        char name[32];
        std::snprintf(name, sizeof(name), "%s_exc1", tag), out.put(name, e1);
        std::snprintf(name, sizeof(name), "%s_exc2", tag), out.put(name, e2);
        std::snprintf(name, sizeof(name), "%s_vxc1", tag), out.put(name, v1);
        std::snprintf(name, sizeof(name), "%s_vxc2", tag), out.put(name, v2);
    }
    return 0;
}

template <class Engine, class Functional>
double runEngineUks(TlSerializeData& param, int iteration, const TlDenseSymmetricMatrix_Lapack& PA,
                    const TlDenseSymmetricMatrix_Lapack& PB, Functional* f, TlDenseSymmetricMatrix_Lapack* FA,
                    TlDenseSymmetricMatrix_Lapack* FB) {
    param["num_of_iterations"] = iteration;
    Engine e(&param);
    return e.calcXCIntegForFockAndEnergy(PA, PB, f, FA, FB);
}

// Open-shell drop-in check: both classes' P_A, P_B overloads for two SCF iterations
// (halves of P_A and P_B, the second with xc-update), through the grid-matrix files.
int runDropinUks(const Case& c, const char* outPath) {
    TlSerializeData param = makeParam(c);
    param["method"] = "uks";
    const TlOrbitalInfo orbProbe(param["coordinates"], param["basis_set"]);
    const int N = orbProbe.getNumOfOrbitals();
    param["num_of_AOs"] = N;
    param["xc-update"] = "yes";
    param["control"]["file_base_name"]["grid_matrix"] = "grid_%s.mat";
    const std::string fn = c.get("functional", "SVWN");
    const bool gga = isGGA(fn);
    const long npts = std::atol(c.get("npts", "0").c_str());
    const int ncol = gga ? 13 : 7;
    const std::vector<double> grid = readDoubles(c.get("grid_file"), (size_t)npts * 5);
    const std::vector<double> P = readDoubles(c.get("density_file"), (size_t)N * N);
    const std::vector<double> Pb = readDoubles(c.get("density_file_b"), (size_t)N * N);
    TlDenseGeneralMatrix_Lapack gridMat(npts, ncol);
    for (long i = 0; i < npts; ++i)
        for (int k = 0; k < 5; ++k) gridMat.set(i, k, grid[5 * i + k]);
    TlDenseSymmetricMatrix_Lapack PA2(N), PB2(N);
    for (int i = 0; i < N; ++i)
        for (int j = 0; j <= i; ++j) PA2.set(i, j, 0.5 * P[(size_t)i * N + j]), PB2.set(i, j, 0.5 * Pb[(size_t)i * N + j]);
    Out out(outPath);
    for (int engine = 0; engine < 2; ++engine) {
        GridFileWriter(&param).save(0, gridMat);
        double e[2] = {0, 0};
        std::vector<TlDenseSymmetricMatrix_Lapack> FA(2, TlDenseSymmetricMatrix_Lapack(N)), FB(FA);
        for (int it = 0; it < 2; ++it) {
            if (gga) {
                DfFunctional_GGA* f = makeGGA(fn);
                e[it] = engine ? runEngineUks<DfCalcGridX_B200>(param, it + 1, PA2, PB2, f, &FA[it], &FB[it])
                               : runEngineUks<DfCalcGridX>(param, it + 1, PA2, PB2, f, &FA[it], &FB[it]);
                delete f;
            } else {
                DfFunctional_LDA* f = makeLDA(fn);
                e[it] = engine ? runEngineUks<DfCalcGridX_B200>(param, it + 1, PA2, PB2, f, &FA[it], &FB[it])
                               : runEngineUks<DfCalcGridX>(param, it + 1, PA2, PB2, f, &FA[it], &FB[it]);
                delete f;
            }
        }
        const char* tag = engine ? "b200" : "ref";
        for (int it = 0; it < 2; ++it) {
            std::vector<double> va((size_t)N * N), vb((size_t)N * N);
            for (int i = 0; i < N; ++i)
                for (int j = 0; j < N; ++j) va[(size_t)i * N + j] = FA[it].get(i, j), vb[(size_t)i * N + j] = FB[it].get(i, j);
            char name[32];
            std::snprintf(name, sizeof(name), "%s_exc%d", tag, it + 1), out.put(name, e[it]);
            std::snprintf(name, sizeof(name), "%s_vxca%d", tag, it + 1), out.put(name, va);
            std::snprintf(name, sizeof(name), "%s_vxcb%d", tag, it + 1), out.put(name, vb);
        }
    }
    return 0;
}

// The XC nuclear gradient through both classes' energyGradient (each builds the
// SG-1 gradient grid itself), then DfCalcGridX_B200 with the grid-weight term on.
// The grid matrix of iteration 0 (DfObject keeps its loader protected).
struct GridMatrixReader : public DfObject {
    explicit GridMatrixReader(TlSerializeData* p) : DfObject(p) {}
    TlDenseGeneralMatrix_Lapack read() { return this->getGridMatrix<TlDenseGeneralMatrix_Lapack>(0); }
};

std::vector<double> rowMajor(const TlDenseGeneralMatrix_Lapack& G) {
    std::vector<double> v;
    for (TlMatrixObject::index_type i = 0; i < G.getNumOfRows(); ++i)
        for (TlMatrixObject::index_type j = 0; j < G.getNumOfCols(); ++j) v.push_back(G.get(i, j));
    return v;
}

// The grid producer: the reference's DfGenerateGrid::dfGrdMain, then DfGenerateGrid_B200's,
// each writing the grid matrix of iteration 0 (read back after each).
int runDropinGenGrid(const Case& c, const char* outPath) {
    TlSerializeData param = makeParam(c);
    const TlOrbitalInfo orbProbe(param["coordinates"], param["basis_set"]);
    param["num_of_AOs"] = orbProbe.getNumOfOrbitals();
    Out out(outPath);
    {
        DfGenerateGrid g(&param);
        g.dfGrdMain();
        const TlDenseGeneralMatrix_Lapack G = GridMatrixReader(&param).read();
        out.put("ref_grid", rowMajor(G));
        out.put("ref_ncol", (double)G.getNumOfCols());
    }
    {
        DfGenerateGrid_B200 g(&param);
        g.dfGrdMain();
        const TlDenseGeneralMatrix_Lapack G = GridMatrixReader(&param).read();
        out.put("b200_grid", rowMajor(G));
        out.put("b200_ncol", (double)G.getNumOfCols());
    }
    return 0;
}

// gridDensity through both classes; the B200 class also through its batched form.
int runDropinDensity(const Case& c, const char* outPath) {
    TlSerializeData param = makeParam(c);
    const TlOrbitalInfo orbProbe(param["coordinates"], param["basis_set"]);
    const int N = orbProbe.getNumOfOrbitals();
    param["num_of_AOs"] = N;
    const int npts = std::atoi(c.get("npts").c_str());
    const std::vector<double> xyz = readDoubles(c.get("points_file"), (size_t)npts * 3);
    const TlDenseSymmetricMatrix_Lapack P = readSymmetric(c, N);
    Out out(outPath);
    out.put("ref_rho", referenceDensities(&param, P, xyz));
    DfCalcGridX_B200 b(&param);
    std::vector<TlPosition> pts;
    std::vector<double> one(npts, 0.0);
    for (int k = 0; k < npts; ++k) {
        pts.emplace_back(xyz[3 * k], xyz[3 * k + 1], xyz[3 * k + 2]);
        if (k < 8) b.gridDensity(P, pts.back(), &one[k]);
    }
    out.put("b200_rho", b.gridDensities(P, pts));
    out.put("b200_rho_single", std::vector<double>(one.begin(), one.begin() + std::min(npts, 8)));
    return 0;
}

int runDropinGrad(const Case& c, const char* outPath) {
    TlSerializeData param = makeParam(c);
    const TlOrbitalInfo orbProbe(param["coordinates"], param["basis_set"]);
    const int N = orbProbe.getNumOfOrbitals();
    param["num_of_AOs"] = N;
    const int natom = (int)c.atomSym.size();
    const std::string fn = c.get("functional", "SVWN");
    const std::vector<double> P = readDoubles(c.get("density_file"), (size_t)N * N);
    TlDenseSymmetricMatrix_Lapack PA(N);
    for (int i = 0; i < N; ++i)
        for (int j = 0; j <= i; ++j) PA.set(i, j, P[(size_t)i * N + j]);
    Out out(outPath);
    for (int engine = 0; engine < 3; ++engine) {
        if (engine == 2) param["xc_gradient/weight_term"] = "yes";
        TlDenseGeneralMatrix_Lapack G;
        if (isGGA(fn)) {
            DfFunctional_GGA* f = makeGGA(fn);
            if (engine == 0) {
                DfCalcGridX e(&param);
                G = e.energyGradient(PA, f);
            } else {
                DfCalcGridX_B200 e(&param);
                G = e.energyGradient(PA, f);
            }
            delete f;
        } else {
            DfFunctional_LDA* f = makeLDA(fn);
            if (engine == 0) {
                DfCalcGridX e(&param);
                G = e.energyGradient(PA, f);
            } else {
                DfCalcGridX_B200 e(&param);
                G = e.energyGradient(PA, f);
            }
            delete f;
        }
        std::vector<double> g(3 * (size_t)natom);
        for (int a = 0; a < natom; ++a)
            for (int k = 0; k < 3; ++k) g[3 * a + k] = G.get(a, k);
        out.put(engine == 0 ? "ref_grad" : engine == 1 ? "b200_grad" : "b200_grad_weight_on", g);
    }
    return 0;
}
#endif

}  // namespace

int main(int argc, char** argv) {
    if (argc != 4) {
        std::fprintf(stderr, "usage: %s xc|grid|func <case.txt> <out.bin>\n", argv[0]);
        return 2;
    }
    TlLogging::getInstance().setLevel(TlLogging::TL_WARN, TlLogging::TL_WARN);
    const std::string mode = argv[1];
    if (mode == "lebedev") return runLebedev(argv[3]);
    const Case c = readCase(argv[2]);
    if (mode == "xc") return runXc(c, argv[3]);
    if (mode == "grid") return runGrid(c, argv[3]);
    if (mode == "func") return runFunc(c, argv[3]);
    if (mode == "grad") return runGrad(c, argv[3]);
    if (mode == "density") return runDensity(c, argv[3]);
#ifdef PDFXC_DROPIN
    if (mode == "dropin_density") return runDropinDensity(c, argv[3]);
    if (mode == "dropin_gengrid") return runDropinGenGrid(c, argv[3]);
    if (mode == "dropin") return runDropin(c, argv[3]);
    if (mode == "dropin_grad") return runDropinGrad(c, argv[3]);
    if (mode == "dropin_uks") return runDropinUks(c, argv[3]);
#endif
    std::fprintf(stderr, "unknown mode %s\n", argv[1]);
    return 2;
}
