"""B200-native grid exchange-correlation quadrature for ProteinDF (DfCalcGridX).

The compute path is libpdfxc.so (hand-written sm_100a CUDA behind the C ABI
declared in include/pdfxc.h). This package holds its Python front end
(proteindf_b200.xc), a mirror of the reference's DfCalcGridX interface
(proteindf_b200.dfcalcgridx), and host helpers that build the inputs
(basis tables, atom-centred grids, seeded synthetic systems).
"""
from .xc import XcEngine, FUNCTIONALS, PRECISION, load_library  # noqa: F401
