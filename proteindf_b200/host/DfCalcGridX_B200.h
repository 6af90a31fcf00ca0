// DfCalcGridX_B200: the drop-in for ProteinDF's DfCalcGridX on one B200.
//
// It derives from the reference class so that it keeps DfObject's parameter
// and file plumbing (iteration number, xc-update, grid.mat) and the orbital
// table, and it re-declares the closed-shell entry points the SCF driver
// reaches through DfXCFunctional::getFxc<SymmetricMatrix, DfCalcGridClass>
// (src/libpdf/DfXCFunctional.h:134-244):
//
//   double calcXCIntegForFockAndEnergy(const TlDenseSymmetricMatrix_Lapack& P_A,
//                                      DfFunctional_LDA* / DfFunctional_GGA*,
//                                      TlDenseSymmetricMatrix_Lapack* F_A);
//
// (src/libpdf/DfCalcGridX.h:194-210), and the XC nuclear gradient the force
// code reaches through DfForce::calcForceFromPureXC (src/libpdf/DfForce.cpp:366-410):
//
//   TlDenseGeneralMatrix_Lapack energyGradient(const TlDenseSymmetricMatrix_Lapack& P_A,
//                                              DfFunctional_LDA* / DfFunctional_GGA*);
//
// (src/libpdf/DfCalcGridX.h:81-88). The computation runs in libpdfxc
// (include/pdfxc.h). The side effects are the reference's: F_A is accumulated
// into, the grid matrix of the previous iteration is read and the one of this
// iteration is written with the new rho / grad rho columns
// (src/libpdf/DfCalcGridX.cpp:1816-1860), so DfXCFunctional::checkGridAccuracy
// and xc-update restarts keep working.
//
// Build: compile this file inside ProteinDF (it includes the reference's
// headers) and link libpdfxc.so.
#ifndef DFCALCGRIDX_B200_H
#define DFCALCGRIDX_B200_H

#include <vector>

#include "DfCalcGridX.h"
#include "pdfxc.h"

class DfCalcGridX_B200 : public DfCalcGridX {
   public:
    explicit DfCalcGridX_B200(TlSerializeData* pPdfParam, int device = 0,
                              int precision = PDFXC_PRECISION_FP64);
    virtual ~DfCalcGridX_B200();

    double calcXCIntegForFockAndEnergy(const TlDenseSymmetricMatrix_Lapack& P_A,
                                       DfFunctional_LDA* pFunctional,
                                       TlDenseSymmetricMatrix_Lapack* pF_A);
    double calcXCIntegForFockAndEnergy(const TlDenseSymmetricMatrix_Lapack& P_A,
                                       DfFunctional_GGA* pFunctional,
                                       TlDenseSymmetricMatrix_Lapack* pF_A);
    // open shell (src/libpdf/DfCalcGridX.h:198-210): F_A, F_B accumulated into; the grid
    // matrix carries rho_A and rho_B columns (LDA 7, GGA 13 columns)
    double calcXCIntegForFockAndEnergy(const TlDenseSymmetricMatrix_Lapack& P_A,
                                       const TlDenseSymmetricMatrix_Lapack& P_B,
                                       DfFunctional_LDA* pFunctional,
                                       TlDenseSymmetricMatrix_Lapack* pF_A,
                                       TlDenseSymmetricMatrix_Lapack* pF_B);
    double calcXCIntegForFockAndEnergy(const TlDenseSymmetricMatrix_Lapack& P_A,
                                       const TlDenseSymmetricMatrix_Lapack& P_B,
                                       DfFunctional_GGA* pFunctional,
                                       TlDenseSymmetricMatrix_Lapack* pF_A,
                                       TlDenseSymmetricMatrix_Lapack* pF_B);

    // XC nuclear gradient, natom x 3, on the reference's own gradient grid
    // (DfGenerateGrid::getGrids, SG-1, built on the host as the reference builds
    // it). The result is the reference's: the AO-centre term (its grid-weight
    // term is identically zero, see pdfxc_xc_gradient). With the parameter
    // "xc_gradient/weight_term" = "yes" the Becke grid-weight derivative is added.
    TlDenseGeneralMatrix_Lapack energyGradient(const TlDenseSymmetricMatrix_Lapack& P_A,
                                               DfFunctional_LDA* pFunctional);
    TlDenseGeneralMatrix_Lapack energyGradient(const TlDenseSymmetricMatrix_Lapack& P_A,
                                               DfFunctional_GGA* pFunctional);

    // rho(r) = phi(r)^T P phi(r) at one point (DfCalcGridX::gridDensity, src/libpdf/DfCalcGridX.cpp:1038-1044)
    // and at many points in one device call, the loop of TlDensField::makeDensFld
    // (src/tools/TlDensField.cpp:35-53); the build grid and its stored densities are untouched
    void gridDensity(const TlDenseSymmetricMatrix_Lapack& P, const TlPosition& gridPosition, double* pRho);
    std::vector<double> gridDensities(const TlDenseSymmetricMatrix_Lapack& P, const std::vector<TlPosition>& grids);

    // sum_i w_i rho_s(r_i) of the last build (DfCalcGridX::getWholeDensity)
    double lastElectronCountAlpha() const { return nelecAlpha_; }
    double lastElectronCountBeta() const { return nelecBeta_; }

   protected:
    double build(const TlDenseSymmetricMatrix_Lapack& P_A, int functionalId, bool gga,
                 TlDenseSymmetricMatrix_Lapack* pF_A);
    double buildOpenShell(const TlDenseSymmetricMatrix_Lapack& P_A, const TlDenseSymmetricMatrix_Lapack& P_B,
                          int functionalId, bool gga, TlDenseSymmetricMatrix_Lapack* pF_A,
                          TlDenseSymmetricMatrix_Lapack* pF_B);
    void loadGrid(const TlDenseGeneralMatrix_Lapack& gridMat);
    static int functionalId(DfFunctional_LDA* f);
    static int functionalId(DfFunctional_GGA* f);
    TlDenseGeneralMatrix_Lapack gradient(const TlDenseSymmetricMatrix_Lapack& P_A, int functionalId);

   private:
    pdfxc_ctx* ctx_ = nullptr;
    pdfxc_ctx* gradCtx_ = nullptr;  // the gradient's own grid
    int device_ = 0;
    // the system as given to libpdfxc, the gradient grid's single-centre weights and Becke radii
    std::vector<double> sysXyz_, pExp_, pCoef_, gradWsingle_, gradRadius_;
    std::vector<int> sysZ_, shAtom_, shL_, shNprim_;
    bool gradSizeAdjust_ = true;
    bool gridLoaded_ = false;
    double nelecAlpha_ = 0.0;
    double nelecBeta_ = 0.0;
};

#endif  // DFCALCGRIDX_B200_H
