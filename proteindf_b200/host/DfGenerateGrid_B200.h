// DfGenerateGrid_B200: the grid producer of ProteinDF (DfGenerateGrid::dfGrdMain,
// src/libpdf/DfGenerateGrid.cpp:254-266, generateGrid :730-768) on one B200.
//
// It derives from the reference class, so that the parameter set is read exactly as the
// reference reads it (grid type, radial shells and method, Gauss-Chebyshev map, angular
// order and pruning, partition method, atomic size adjustment, weight cut-off; the
// orientation matrix O of getOMatrix; the Lebedev tables of TlLebedevGrid), and generates
// the grid with pdfxc_generate_grid: points, single-centre weights and partition weights
// on the device. dfGrdMain() writes the same grid matrix (x, y, z, weight, atom index and
// zeroed density columns, iteration 0) through DfObject::saveGridMatrix, so DfCalcGridX
// and DfCalcGridX_B200 read it as they read the reference's. Rows are atom after atom in
// atom order (the reference's OpenMP loop over atoms appends them in completion order).
//
// Build: compile this file inside ProteinDF (it includes the reference's headers) and link
// libpdfxc.so.
#ifndef DFGENERATEGRID_B200_H
#define DFGENERATEGRID_B200_H

#include <cstdint>

#include "DfGenerateGrid.h"
#include "pdfxc.h"

class DfGenerateGrid_B200 : public DfGenerateGrid {
   public:
    explicit DfGenerateGrid_B200(TlSerializeData* pPdfParam, int device = 0);
    virtual ~DfGenerateGrid_B200();

    // generates the grid on the device and saves the grid matrix of iteration 0
    int dfGrdMain();

    // points of the last generated grid
    int64_t numOfGridPoints() const { return npts_; }

   private:
    pdfxc_ctx* ctx_ = nullptr;
    int64_t npts_ = 0;
};

#endif  // DFGENERATEGRID_B200_H
