// Oracle (test infrastructure): elastic::reactions, crates/fem/src/elastic.rs:772-839, as
// written there: K u over all unknowns (Csr::mul, sparse.rs:96-105), then one pass over the
// unknowns in increasing order, adding r = (K u)_i - f_i of each fixed unknown to the total of
// its component, to the gross magnitude and to the force of its owner (a fixed face set's
// Reaction or a point support's point_force), then the imbalance (elastic.rs:827-831).
#include <cmath>

#include "oracle.hpp"

namespace orc {

void reactions(const Csr& k, const double* u, const double* force, const uint8_t* fixed,
               const uint32_t* owner, size_t nloads, const double applied[3], double gross,
               double* load_force, double total[3], double* gross_out, double* imbalance) {
    vector<double> ku(k.n, 0.0);
    k.mul(u, ku.data());
    for (size_t q = 0; q < 3 * nloads; ++q) load_force[q] = 0.0;
    for (int c = 0; c < 3; ++c) total[c] = applied[c];
    for (size_t i = 0; i < k.n; ++i) {
        if (!fixed[i]) continue;
        double r = ku[i] - force[i];
        total[i % 3] += r;
        gross += std::fabs(r);
        size_t o = owner[i];
        if (o < nloads) load_force[3 * o + i % 3] += r;
    }
    // fold(0.0, f64::max) over |total|: f64::max returns the other operand when one is NaN.
    double m = 0.0;
    for (int c = 0; c < 3; ++c) {
        double a = std::fabs(total[c]);
        if (!(a <= m) && a == a) m = a;
    }
    *gross_out = gross;
    *imbalance = gross > 0.0 ? m / gross : 0.0;
}

}  // namespace orc
