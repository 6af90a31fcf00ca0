// The system as libpdfxc takes it (pdfxc_set_system), read from the reference's orbital
// table: a shell starts at its first component (basis type L*L); exponents and normalised
// coefficients are TlOrbitalInfo's own (src/libpdf/TlOrbitalInfoObject.cpp:38-99).
#ifndef PDFXC_SYSTEM_H
#define PDFXC_SYSTEM_H

#include <vector>

#include "TlOrbitalInfo.h"
#include "pdfxc.h"

struct PdfxcSystem {
    std::vector<double> xyz, pExp, pCoef;
    std::vector<int> z, shAtom, shL, shNprim;

    explicit PdfxcSystem(const TlOrbitalInfo& orb) {
        const int natom = orb.getNumOfAtoms();
        xyz.assign(3 * natom, 0.0);
        z.assign(natom, 0);
        const int nao = orb.getNumOfOrbitals();
        for (int ao = 0; ao < nao; ++ao) {
            const int a = orb.getAtomIndex(ao);
            const TlPosition r = orb.getPosition(ao);
            xyz[3 * a] = r.x(), xyz[3 * a + 1] = r.y(), xyz[3 * a + 2] = r.z();
            z[a] = (int)orb.getAtomCharge(ao);
            const int L = orb.getShellType(ao);
            if (orb.getBasisType(ao) != L * L) continue;  // not the first component
            shAtom.push_back(a);
            shL.push_back(L);
            const int np = orb.getCgtoContraction(ao);
            shNprim.push_back(np);
            for (int k = 0; k < np; ++k) {
                pExp.push_back(orb.getExponent(ao, k));
                pCoef.push_back(orb.getCoefficient(ao, k));
            }
        }
    }

    pdfxc_status setOn(pdfxc_ctx* ctx) const {
        return pdfxc_set_system(ctx, (int)z.size(), xyz.data(), z.data(), (int)shAtom.size(), shAtom.data(),
                                shL.data(), shNprim.data(), pExp.data(), pCoef.data());
    }
};

#endif  // PDFXC_SYSTEM_H
