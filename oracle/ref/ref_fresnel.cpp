/*
 * FresnelDielectric::evaluate (declared in src/filianore/shading/fresnel/fresneldielectric.h)
 * compiled in place of src/filianore/shading/fresnel/fresneldielectric.cpp, whose version
 * swaps its `mutable` etaI/etaT members for exiting rays (fresneldielectric.cpp:12-16), so
 * its answer depends on earlier calls on the same object. This one delegates to the
 * reference's own stateless fresnel_dielectric_evaluation (fresnel/fresnel.h:25-56), which
 * performs the same arithmetic on local copies. Test infrastructure only.
 */
#include "filianore/shading/fresnel/fresneldielectric.h"
#include "filianore/shading/fresnel/fresnel.h"

namespace filianore {

PrincipalSpectrum FresnelDielectric::evaluate(float cosThetaI) const {
    return PrincipalSpectrum(fresnel_dielectric_evaluation(cosThetaI, etaI, etaT));
}

} // namespace filianore
