// DfGenerateGrid_B200: see DfGenerateGrid_B200.h.
#include "DfGenerateGrid_B200.h"

#include <stdexcept>
#include <string>
#include <vector>

#include "TlOrbitalInfo.h"
#include "TlPrdctbl.h"
#include "pdfxc_system.h"

namespace {

void check(pdfxc_status st, pdfxc_ctx* ctx, const char* what) {
    if (st != PDFXC_OK)
        throw std::runtime_error(std::string(what) + " failed: " + (ctx ? pdfxc_last_error(ctx) : "no context"));
}

}  // namespace

DfGenerateGrid_B200::DfGenerateGrid_B200(TlSerializeData* pPdfParam, int device) : DfGenerateGrid(pPdfParam) {
    pdfxc_options opt;
    pdfxc_default_options(&opt);
    check(pdfxc_create(&ctx_, device, &opt), nullptr, "pdfxc_create");
    const TlOrbitalInfo orb((*pPdfParam)["coordinates"], (*pPdfParam)["basis_set"]);
    check(PdfxcSystem(orb).setOn(ctx_), ctx_, "pdfxc_set_system");
}

DfGenerateGrid_B200::~DfGenerateGrid_B200() { pdfxc_destroy(ctx_); }

int DfGenerateGrid_B200::dfGrdMain() {
    const int natom = this->m_nNumOfAtoms;
    // per atom: the radial scale (the SG-1 radii for SG-1, Bragg-Slater otherwise,
    // generateGrid_atom :951-957) and the Becke size-adjustment radius
    // (getCovalentRadiiForBecke, :1958-1968); dummy atoms get no grid (:950-952)
    std::vector<double> radius(natom, 0.0), becke(natom, 0.0);
    for (int a = 0; a < natom; ++a) {
        const int Z = TlPrdctbl::getAtomicNumber(this->flGeometry_.getAtomSymbol(a));
        if (Z == 0) continue;
        radius[a] = this->m_gridType == SG_1 ? this->radiusList_[Z] : TlPrdctbl::getBraggSlaterRadii(Z);
        becke[a] = Z == 1 ? 0.35 : TlPrdctbl::getBraggSlaterRadii(Z);
    }
    // the Lebedev tables of the reference's own TlLebedevGrid
    std::vector<int> orders = this->lebGrd_.getSupportedGridNumber();
    std::vector<double> unit;
    for (int n : orders) {
        std::vector<TlPosition> p;
        std::vector<double> w;
        this->lebGrd_.getGrids(n, &p, &w);
        for (int k = 0; k < n; ++k) unit.insert(unit.end(), {p[k].x(), p[k].y(), p[k].z(), w[k]});
    }
    double O[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) O[3 * i + j] = this->O_.get(i, j);

    pdfxc_grid_params prm{};
    prm.nrad = this->nrgrid;
    prm.nang = this->nOgrid;
    // the reference's private enums, by value: RADIAL_GRID_TYPE {EulerMaclaurin, GaussChebyshev},
    // GC_MAPPING_TYPE {Becke, TA, KK}, PARTITIONING_METHOD {Becke, SSWeight} (DfGenerateGrid.h:84-88)
    prm.radial = static_cast<int>(this->radialGridType_) == 1 ? PDFXC_RADIAL_GC : PDFXC_RADIAL_EM;
    prm.mapping = static_cast<int>(this->GC_mappingType_);
    prm.pruning = this->m_gridType == SG_1 ? PDFXC_PRUNE_SG1 : (this->isPruning_ ? PDFXC_PRUNE_MHL : PDFXC_PRUNE_NONE);
    prm.partition = static_cast<int>(this->partitioningMethod_) == 1 ? PDFXC_PARTITION_SS : PDFXC_PARTITION_BECKE;
    prm.size_adjust = this->isAtomicSizeAdjustments_ ? 1 : 0;
    prm.weight_cutoff = this->weightCutoff_;
    prm.atom_radius = radius.data();
    prm.becke_radius = becke.data();
    prm.n_orders = (int)orders.size();
    prm.orders = orders.data();
    prm.unit_grids = unit.data();
    prm.orientation = O;
    check(pdfxc_generate_grid(ctx_, &prm, &npts_), ctx_, "pdfxc_generate_grid");

    std::vector<double> xyzw(4 * (size_t)npts_);
    std::vector<int> atom((size_t)npts_);
    check(pdfxc_get_grid(ctx_, xyzw.data(), atom.data()), ctx_, "pdfxc_get_grid");
    TlDenseGeneralMatrix_Lapack grid(npts_, this->numOfColsOfGrdMat_);
    for (int64_t i = 0; i < npts_; ++i) {
        for (int k = 0; k < 4; ++k) grid.set(i, k, xyzw[4 * i + k]);
        grid.set(i, 4, atom[i]);
    }
    this->saveGridMatrix(0, grid);
    return 0;
}
