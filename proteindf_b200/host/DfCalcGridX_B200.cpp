// DfCalcGridX_B200: see DfCalcGridX_B200.h.
#include "DfCalcGridX_B200.h"

#include <stdexcept>
#include <string>

#include "DfFunctional_B3LYP.h"
#include "DfFunctional_B88LYP.h"
#include "DfFunctional_Becke88.h"
#include "DfFunctional_HFS.h"
#include "DfFunctional_SVWN.h"
#include "DfGenerateGrid.h"
#include "TlPrdctbl.h"
#include "TlUtils.h"
#include "pdfxc_system.h"

namespace {

void check(pdfxc_status st, pdfxc_ctx* ctx, const char* what) {
    if (st != PDFXC_OK)
        throw std::runtime_error(std::string(what) + " failed: " + (ctx ? pdfxc_last_error(ctx) : "no context"));
}

}  // namespace

DfCalcGridX_B200::DfCalcGridX_B200(TlSerializeData* pPdfParam, int device, int precision)
    : DfCalcGridX(pPdfParam), device_(device) {
    pdfxc_options opt;
    pdfxc_default_options(&opt);
    opt.precision = precision;
    opt.rho_cutoff = this->inputtedDensityCutoffValue_;  // xc-density-threshold
    check(pdfxc_create(&ctx_, device, &opt), nullptr, "pdfxc_create");

    const PdfxcSystem sys(this->m_tlOrbInfo);
    check(sys.setOn(ctx_), ctx_, "pdfxc_set_system");
    sysXyz_ = sys.xyz, sysZ_ = sys.z, shAtom_ = sys.shAtom, shL_ = sys.shL, shNprim_ = sys.shNprim;
    pExp_ = sys.pExp, pCoef_ = sys.pCoef;
}

DfCalcGridX_B200::~DfCalcGridX_B200() {
    pdfxc_destroy(gradCtx_);
    pdfxc_destroy(ctx_);
}

std::vector<double> DfCalcGridX_B200::gridDensities(const TlDenseSymmetricMatrix_Lapack& P,
                                                    const std::vector<TlPosition>& grids) {
    const int n = this->m_nNumOfAOs;
    std::vector<double> full((size_t)n * n);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j <= i; ++j) full[(size_t)i * n + j] = full[(size_t)j * n + i] = P.get(i, j);
    std::vector<double> xyz(3 * grids.size()), rho(grids.size(), 0.0);
    for (size_t k = 0; k < grids.size(); ++k)
        xyz[3 * k] = grids[k].x(), xyz[3 * k + 1] = grids[k].y(), xyz[3 * k + 2] = grids[k].z();
    check(pdfxc_density(ctx_, full.data(), (int64_t)grids.size(), xyz.data(), rho.data()), ctx_, "pdfxc_density");
    return rho;
}

void DfCalcGridX_B200::gridDensity(const TlDenseSymmetricMatrix_Lapack& P, const TlPosition& gridPosition,
                                   double* pRho) {
    *pRho = this->gridDensities(P, std::vector<TlPosition>(1, gridPosition))[0];
}

TlDenseGeneralMatrix_Lapack DfCalcGridX_B200::energyGradient(const TlDenseSymmetricMatrix_Lapack& P_A,
                                                             DfFunctional_LDA* pFunctional) {
    return this->gradient(P_A, functionalId(pFunctional));
}

TlDenseGeneralMatrix_Lapack DfCalcGridX_B200::energyGradient(const TlDenseSymmetricMatrix_Lapack& P_A,
                                                             DfFunctional_GGA* pFunctional) {
    return this->gradient(P_A, functionalId(pFunctional));
}

TlDenseGeneralMatrix_Lapack DfCalcGridX_B200::gradient(const TlDenseSymmetricMatrix_Lapack& P_A, int fn) {
    TlSerializeData& param = *(this->pPdfParam_);
    const int natom = (int)sysZ_.size();
    if (!gradCtx_) {
        pdfxc_options opt;
        pdfxc_default_options(&opt);
        opt.rho_cutoff = this->inputtedDensityCutoffValue_;
        check(pdfxc_create(&gradCtx_, device_, &opt), nullptr, "pdfxc_create");
        check(pdfxc_set_system(gradCtx_, natom, sysXyz_.data(), sysZ_.data(), (int)shAtom_.size(), shAtom_.data(),
                               shL_.data(), shNprim_.data(), pExp_.data(), pCoef_.data()),
              gradCtx_, "pdfxc_set_system");
        // the grid energyGradient_part integrates on (src/libpdf/DfCalcGridX.cpp:1119-1121):
        // per atom, single-centre weight times Becke partition weight
        DfGenerateGrid gen(this->pPdfParam_);
        std::vector<double> xyzw;
        std::vector<int> atom;
        gradWsingle_.clear();
        for (int a = 0; a < natom; ++a) {
            std::vector<TlPosition> pts;
            std::vector<double> ws, wp;
            gen.getGrids(a, &pts, &ws, &wp);
            for (size_t k = 0; k < pts.size(); ++k) {
                xyzw.insert(xyzw.end(), {pts[k].x(), pts[k].y(), pts[k].z(), ws[k] * wp[k]});
                atom.push_back(a);
                gradWsingle_.push_back(ws[k]);
            }
        }
        check(pdfxc_set_grid(gradCtx_, (int64_t)atom.size(), xyzw.data(), atom.data()), gradCtx_, "pdfxc_set_grid");
        // Becke radii and size adjustment as DfGenerateGrid sets them
        // (src/libpdf/DfGenerateGrid.cpp:120-160, :1958-1968)
        gradRadius_.assign(natom, 0.0);
        for (int a = 0; a < natom; ++a)
            gradRadius_[a] = sysZ_[a] == 1 ? 0.35 : TlPrdctbl::getBraggSlaterRadii(sysZ_[a]);
        const std::string gt = TlUtils::toUpper(param["xc-potential/grid-type"].getStr());
        gradSizeAdjust_ = !(gt == "SG-1" || gt == "SG1");
        if (param["grid/atomic_size_adjustments"].getStr() != "")
            gradSizeAdjust_ = param["grid/atomic_size_adjustments"].getBoolean();
    }
    const bool weightTerm = TlUtils::toUpper(param["xc_gradient/weight_term"].getStr()) == "YES";
    const int n = this->m_nNumOfAOs;
    std::vector<double> P((size_t)n * n);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j <= i; ++j) P[(size_t)i * n + j] = P[(size_t)j * n + i] = P_A.get(i, j);
    std::vector<double> go(3 * (size_t)natom, 0.0), gw(3 * (size_t)natom, 0.0);
    double exc = 0.0;
    check(pdfxc_xc_gradient(gradCtx_, fn, P.data(), weightTerm ? gradWsingle_.data() : nullptr, gradRadius_.data(),
                            gradSizeAdjust_ ? 1 : 0, go.data(), weightTerm ? gw.data() : nullptr, &exc),
          gradCtx_, "pdfxc_xc_gradient");
    TlDenseGeneralMatrix_Lapack G(natom, 3);
    for (int a = 0; a < natom; ++a)
        for (int k = 0; k < 3; ++k) G.set(a, k, go[3 * a + k] + gw[3 * a + k]);
    return G;
}

int DfCalcGridX_B200::functionalId(DfFunctional_LDA* f) {
    if (dynamic_cast<DfFunctional_SVWN*>(f)) return PDFXC_SVWN;
    if (dynamic_cast<DfFunctional_HFS*>(f)) return PDFXC_HFS;
    throw std::runtime_error("DfCalcGridX_B200: unsupported LDA functional");
}

int DfCalcGridX_B200::functionalId(DfFunctional_GGA* f) {
    if (dynamic_cast<DfFunctional_B3LYP*>(f)) return PDFXC_B3LYP;
    if (dynamic_cast<DfFunctional_B88LYP*>(f)) return PDFXC_BLYP;
    if (dynamic_cast<DfFunctional_Becke88*>(f)) return PDFXC_HFB;
    throw std::runtime_error("DfCalcGridX_B200: unsupported GGA functional");
}

double DfCalcGridX_B200::calcXCIntegForFockAndEnergy(const TlDenseSymmetricMatrix_Lapack& P_A,
                                                     DfFunctional_LDA* pFunctional,
                                                     TlDenseSymmetricMatrix_Lapack* pF_A) {
    return this->build(P_A, functionalId(pFunctional), false, pF_A);
}

double DfCalcGridX_B200::calcXCIntegForFockAndEnergy(const TlDenseSymmetricMatrix_Lapack& P_A,
                                                     DfFunctional_GGA* pFunctional,
                                                     TlDenseSymmetricMatrix_Lapack* pF_A) {
    return this->build(P_A, functionalId(pFunctional), true, pF_A);
}

double DfCalcGridX_B200::calcXCIntegForFockAndEnergy(const TlDenseSymmetricMatrix_Lapack& P_A,
                                                     const TlDenseSymmetricMatrix_Lapack& P_B,
                                                     DfFunctional_LDA* pFunctional,
                                                     TlDenseSymmetricMatrix_Lapack* pF_A,
                                                     TlDenseSymmetricMatrix_Lapack* pF_B) {
    return this->buildOpenShell(P_A, P_B, functionalId(pFunctional), false, pF_A, pF_B);
}

double DfCalcGridX_B200::calcXCIntegForFockAndEnergy(const TlDenseSymmetricMatrix_Lapack& P_A,
                                                     const TlDenseSymmetricMatrix_Lapack& P_B,
                                                     DfFunctional_GGA* pFunctional,
                                                     TlDenseSymmetricMatrix_Lapack* pF_A,
                                                     TlDenseSymmetricMatrix_Lapack* pF_B) {
    return this->buildOpenShell(P_A, P_B, functionalId(pFunctional), true, pF_A, pF_B);
}

// points, weights and owner atoms of the grid matrix, once
void DfCalcGridX_B200::loadGrid(const TlDenseGeneralMatrix_Lapack& gridMat) {
    if (gridLoaded_) return;
    const int64_t npts = gridMat.getNumOfRows();
    std::vector<double> xyzw(4 * npts);
    std::vector<int> atom(npts);
    for (int64_t i = 0; i < npts; ++i) {
        for (int k = 0; k < 4; ++k) xyzw[4 * i + k] = gridMat.get(i, k);
        atom[i] = (int)(gridMat.get(i, GM_ATOM_INDEX) + 0.5);
    }
    check(pdfxc_set_grid(ctx_, npts, xyzw.data(), atom.data()), ctx_, "pdfxc_set_grid");
    gridLoaded_ = true;
}

double DfCalcGridX_B200::buildOpenShell(const TlDenseSymmetricMatrix_Lapack& P_A,
                                        const TlDenseSymmetricMatrix_Lapack& P_B, int fn, bool gga,
                                        TlDenseSymmetricMatrix_Lapack* pF_A, TlDenseSymmetricMatrix_Lapack* pF_B) {
    // grid-matrix columns of the open shell: rho_A (grad rho_A) then rho_B (grad rho_B)
    // from column GM_LDA_RHO_ALPHA = GM_GGA_RHO_ALPHA (src/libpdf/DfCalcGridX.h:35-54)
    TlDenseGeneralMatrix_Lapack gridMat =
        DfObject::getGridMatrix<TlDenseGeneralMatrix_Lapack>(this->m_nIteration - 1);
    const int64_t npts = gridMat.getNumOfRows();
    const int nc = gga ? 8 : 2;
    this->loadGrid(gridMat);
    const bool incremental = (this->m_nIteration > 1) && this->m_bIsUpdateXC;
    if (incremental) {
        std::vector<double> rho(nc * npts);
        for (int64_t i = 0; i < npts; ++i)
            for (int k = 0; k < nc; ++k) rho[nc * i + k] = gridMat.get(i, GM_LDA_RHO_ALPHA + k);
        check(pdfxc_set_rho_uks(ctx_, gga ? 1 : 0, rho.data()), ctx_, "pdfxc_set_rho_uks");
    }
    const int n = this->m_nNumOfAOs;
    std::vector<double> PA((size_t)n * n), PB((size_t)n * n), FA((size_t)n * n, 0.0), FB((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j <= i; ++j) {
            PA[(size_t)i * n + j] = PA[(size_t)j * n + i] = P_A.get(i, j);
            PB[(size_t)i * n + j] = PB[(size_t)j * n + i] = P_B.get(i, j);
        }
    double exc = 0.0;
    check(pdfxc_build_vxc_uks(ctx_, fn, PA.data(), PB.data(), incremental ? 1 : 0, FA.data(), FB.data(), &exc,
                              &nelecAlpha_, &nelecBeta_),
          ctx_, "pdfxc_build_vxc_uks");
    for (int i = 0; i < n; ++i)
        for (int j = 0; j <= i; ++j) pF_A->add(i, j, FA[(size_t)i * n + j]), pF_B->add(i, j, FB[(size_t)i * n + j]);
    std::vector<double> rho(nc * npts);
    check(pdfxc_get_rho_uks(ctx_, gga ? 1 : 0, rho.data()), ctx_, "pdfxc_get_rho_uks");
    for (int64_t i = 0; i < npts; ++i)
        for (int k = 0; k < nc; ++k) gridMat.set(i, GM_LDA_RHO_ALPHA + k, rho[nc * i + k]);
    DfObject::saveGridMatrix(this->m_nIteration, gridMat);
    return exc;
}

double DfCalcGridX_B200::build(const TlDenseSymmetricMatrix_Lapack& P_A, int fn, bool gga,
                               TlDenseSymmetricMatrix_Lapack* pF_A) {
    // the grid matrix of the previous iteration: points, weights and (for
    // xc-update) the accumulated rho columns (DfCalcGridX.cpp:1816-1870)
    TlDenseGeneralMatrix_Lapack gridMat =
        DfObject::getGridMatrix<TlDenseGeneralMatrix_Lapack>(this->m_nIteration - 1);
    const int64_t npts = gridMat.getNumOfRows();
    const int nrho = gga ? 4 : 1;
    this->loadGrid(gridMat);
    const bool incremental = (this->m_nIteration > 1) && this->m_bIsUpdateXC;
    if (incremental) {
        std::vector<double> rho(nrho * npts);
        for (int64_t i = 0; i < npts; ++i)
            for (int k = 0; k < nrho; ++k) rho[nrho * i + k] = gridMat.get(i, GM_LDA_RHO_ALPHA + k);
        check(pdfxc_set_rho(ctx_, gga ? 1 : 0, rho.data()), ctx_, "pdfxc_set_rho");
    }
    const int n = this->m_nNumOfAOs;
    std::vector<double> P((size_t)n * n), F((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j <= i; ++j) P[(size_t)i * n + j] = P[(size_t)j * n + i] = P_A.get(i, j);
    double exc = 0.0;
    check(pdfxc_build_vxc(ctx_, fn, P.data(), incremental ? 1 : 0, F.data(), &exc, &nelecAlpha_), ctx_,
          "pdfxc_build_vxc");
    for (int i = 0; i < n; ++i)
        for (int j = 0; j <= i; ++j) pF_A->add(i, j, F[(size_t)i * n + j]);
    // write this iteration's grid matrix with the new rho columns
    std::vector<double> rho(nrho * npts);
    check(pdfxc_get_rho(ctx_, gga ? 1 : 0, rho.data()), ctx_, "pdfxc_get_rho");
    for (int64_t i = 0; i < npts; ++i)
        for (int k = 0; k < nrho; ++k) gridMat.set(i, GM_LDA_RHO_ALPHA + k, rho[nrho * i + k]);
    DfObject::saveGridMatrix(this->m_nIteration, gridMat);
    return exc;
}
