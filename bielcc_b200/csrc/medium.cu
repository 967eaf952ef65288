// medium.cu — host-side constants of a field evaluation inside a material:
// the absolute permittivity and permeability at a frequency, the wave number,
// the Stratton-Chu multipliers and the incident plane wave, restating
//   MaterialParam::Calc / CalcEps / CalcEpsN / CalcEpsNK / CalcMu / CalcSkinDepth
//       (electrodynamics/material.cpp:60-128),
//   RadiationSource::CalcK (electrodynamics/radiation_source.cpp:159-180),
//   multE = i / (2 pi f eps), multH = i / (2 pi f mu)
//       (examples/field/main0_field_test.cpp:185-199),
//   PlaneWaveFieldE / PlaneWaveFieldH (electrodynamics/incident_field.h:20-59).
// No GPU work. Divergences from the reference, on purpose:
//   * a lossy material (complex eps) gets the complex wave number
//     omega sqrt(eps mu) (Im k > 0, the attenuating branch); the reference's
//     CalcK reads mu as std::complex there while CalcMu always stores a
//     double, so it throws std::bad_variant_access;
//   * a frequency missing from a refractive-index table is an error; the
//     reference's std::map::operator[] inserts n = 0 and continues with eps = 0;
//   * the skin depth of a refractive-index material is 0: the reference's
//     constructors for those leave _sigma uninitialised and CalcSkinDepth
//     reads it.
#include <cmath>
#include <complex>
#include <cstring>

#include "../../include/bielcc_gpu.h"
#include "internal.h"

namespace {

using cd = std::complex<double>;
constexpr double kEps0 = 8.8541878128e-12;  // ED_Constants::eps0 (electrodynamics/constants.h:12)
constexpr double kMu0 = 4 * M_PI * 1e-7;    // ED_Constants::mu0 (constants.h:13)

}  // namespace

extern "C" int bielcc_medium_at(const bielcc_material* mat, double freq, bielcc_medium* out) {
    using namespace bielcc_gpu;
    if (!mat || !out) return set_api_error(BIELCC_ERR_ARG, "null material or medium");
    if (!(freq > 0.) || !std::isfinite(freq)) return set_api_error(BIELCC_ERR_ARG, "frequency must be positive");
    const double omega = 2. * M_PI * freq;
    cd eps;
    double tand = 0.;
    if (mat->dispersion == BIELCC_DISPERSION_REFRACT) {
        if (mat->n_table < 1 || !mat->table) return set_api_error(BIELCC_ERR_ARG, "empty refractive-index table");
        const double* row = nullptr;
        for (int i = 0; i < mat->n_table; i++)
            if (mat->table[3 * i] == freq) row = mat->table + 3 * i;
        if (!row) return set_api_error(BIELCC_ERR_ARG, "frequency not in the refractive-index table");
        const double n = row[1], ka = row[2];
        if (ka == 0.) {  // CalcEpsN
            eps = n * n * kEps0;
            tand = 0.;
        } else {  // CalcEpsNK (its tand = 2 n k eps0, as the reference computes it)
            eps = cd(n * n - ka * ka, 2. * n * ka) * kEps0;
            tand = 2. * n * ka * kEps0;
        }
    } else if (mat->dispersion == BIELCC_DISPERSION_NONE) {  // CalcEps
        if (mat->sigma == 0.) {
            eps = kEps0 * mat->eps_r;
            tand = 0.;
        } else {
            eps = cd(kEps0 * mat->eps_r, mat->sigma / omega);
            tand = mat->sigma / (omega * kEps0 * mat->eps_r);
        }
    } else {
        return set_api_error(BIELCC_ERR_ARG, "unknown dispersion type");
    }
    const double mu = kMu0 * mat->mu_r;  // CalcMu: real
    memset(out, 0, sizeof(*out));
    out->eps[0] = eps.real();
    out->eps[1] = eps.imag();
    out->mu[0] = mu;
    out->mu[1] = 0.;
    // CalcK: gamma = i omega sqrt(eps mu); the principal square root has
    // Re >= 0, and with Im eps >= 0 also Im >= 0, so k = omega sqrt(eps mu)
    // attenuates along its direction of travel
    const cd k = omega * std::sqrt(eps * mu);
    out->k[0] = k.real();
    out->k[1] = k.imag();
    out->k_source = k.real();  // RadiationSource's _k = Im gamma = Re k
    const cd me = cd(0., 1.) / (omega * eps), mh = cd(0., 1.) / (omega * mu);
    out->multE[0] = me.real();
    out->multE[1] = me.imag();
    out->multH[0] = mh.real();
    out->multH[1] = mh.imag();
    out->tand = tand;
    // CalcSkinDepth (only the sigma form, as the reference)
    out->skin_depth = mat->dispersion == BIELCC_DISPERSION_NONE && mat->sigma != 0.
                          ? std::sqrt(2. / (omega * mat->mu_r * kMu0 * mat->sigma))
                          : 0.;
    return BIELCC_OK;
}

extern "C" int bielcc_planewave_in_medium(const bielcc_medium* md, double freq, const double* direction,
                                          const double* e0, int add_E, int add_H, bielcc_planewave* out) {
    using namespace bielcc_gpu;
    if (!md || !direction || !e0 || !out) return set_api_error(BIELCC_ERR_ARG, "null argument");
    if (!(freq > 0.)) return set_api_error(BIELCC_ERR_ARG, "frequency must be positive");
    const double l = std::sqrt(direction[0] * direction[0] + direction[1] * direction[1] +
                               direction[2] * direction[2]);
    if (!(l > 0.)) return set_api_error(BIELCC_ERR_ARG, "zero direction");
    for (int g = 0; g < 3; g++) {
        out->k_vec[g] = md->k_source * direction[g] / l;  // RadiationSource::CalcK: k * ort
        out->e0[g] = e0[g];
    }
    // PlaneWaveFieldH: (k_vec x e0) e^{i k_vec . x} / (2 pi f mu), mu real
    out->h_scale = 1. / (2. * M_PI * freq * md->mu[0]);
    out->add_E = add_E;
    out->add_H = add_H;
    return BIELCC_OK;
}
