// Oracle (test infrastructure): the post-solve recovery of the 10-node tetrahedra. Restates
// the loop of crates/fem/src/elastic_tet.rs:367-427 (the strain and the stress at the 10 points
// of each cell, their mean at each point, the peak of each part), with
// crates/fem/src/tet10.rs:77-87 (the gradients of the 10 functions), tet10.rs:142-169
// (strain_stress), tet10.rs:216-228 (node_coordinates), crates/fem/src/hex.rs:128-139
// (Stiffness::stress), crates/fem/src/elastic.rs:965-1002 (reorder, tensor_strain, mises,
// principal), elastic_tet.rs:164-170 (D alpha of a material) and elastic_tet.rs:482-483 (the
// von Mises stress and the principal stresses of the mean stress at each point).
#include <array>
#include <cmath>
#include <utility>
#include <limits>

#include "oracle.hpp"

namespace orc {

namespace {
// tet10.rs:38 and tet10.rs:41
const int EDGES[6][2] = {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {1, 3}, {2, 3}};
const int SHEAR[3][2] = {{1, 2}, {0, 2}, {0, 1}};
}  // namespace

// tet10.rs:216-228: the volume coordinates of point c of a tetrahedron.
void node_coordinates(int c, double l[4]) {
    for (int k = 0; k < 4; ++k) l[k] = 0.0;
    if (c < 4) {
        l[c] = 1.0;
    } else {
        l[EDGES[c - 4][0]] = 0.5;
        l[EDGES[c - 4][1]] = 0.5;
    }
}

// tet10.rs:142-169. `g` are the gradients of the 4 volume coordinates, `u` the 30 displacements
// (3 point + component), `t` the corner temperature changes. e: engineering strain, s: stress,
// both xx, yy, zz, yz, xz, xy.
void tet10_strain_stress(const Vec3 g[4], const Stiffness& d, const double thermal[3],
                         const double l[4], const double u[30], const double t[4], double e[6],
                         double s[6]) {
    double gr[10][3];
    for (int i = 0; i < 4; ++i)
        for (int k = 0; k < 3; ++k) gr[i][k] = (4.0 * l[i] - 1.0) * g[i][k];
    for (int k = 0; k < 6; ++k) {
        int i = EDGES[k][0], j = EDGES[k][1];
        for (int dd = 0; dd < 3; ++dd) gr[4 + k][dd] = 4.0 * (l[i] * g[j][dd] + l[j] * g[i][dd]);
    }
    for (int a = 0; a < 6; ++a) e[a] = 0.0;
    for (int i = 0; i < 10; ++i) {
        const double* gi = gr[i];
        const double* ui = u + 3 * i;
        for (int a = 0; a < 3; ++a) e[a] += gi[a] * ui[a];
        for (int sh = 0; sh < 3; ++sh) {
            int a = SHEAR[sh][0], b = SHEAR[sh][1];
            e[3 + sh] += gi[a] * ui[b] + gi[b] * ui[a];
        }
    }
    // The Rust float sum starts from -0.0.
    double dt = -0.0;
    for (int c = 0; c < 4; ++c) dt += l[c] * t[c];
    // hex.rs:128-139
    for (int a = 0; a < 3; ++a)
        s[a] = d.normal[a][0] * e[0] + d.normal[a][1] * e[1] + d.normal[a][2] * e[2];
    for (int sh = 0; sh < 3; ++sh) s[3 + sh] = d.shear[sh] * e[3 + sh];
    for (int a = 0; a < 3; ++a) s[a] -= thermal[a] * dt;
}

// elastic.rs:965-983
void reorder_stress(const double s[6], double out[6]) {
    const double r[6] = {s[0], s[1], s[2], s[5], s[3], s[4]};
    for (int i = 0; i < 6; ++i) out[i] = r[i];
}
void tensor_strain(const double e[6], double out[6]) {
    const double r[6] = {e[0], e[1], e[2], 0.5 * e[5], 0.5 * e[3], 0.5 * e[4]};
    for (int i = 0; i < 6; ++i) out[i] = r[i];
}
double mises(const double s[6]) {
    double xx = s[0], yy = s[1], zz = s[2], xy = s[3], yz = s[4], xz = s[5];
    double a = xx - yy, b = yy - zz, c = zz - xx;
    return std::sqrt(0.5 * (a * a + b * b + c * c) + 3.0 * (xy * xy + yz * yz + xz * xz));
}

// elastic.rs:985-1002 (O. K. Smith, Eigenvalues of a symmetric 3 x 3 matrix, Comm. ACM 4
// (1961) 168), largest first.
void principal(const double s[6], double out[3]) {
    double xx = s[0], yy = s[1], zz = s[2], xy = s[3], yz = s[4], xz = s[5];
    double q = (xx + yy + zz) / 3.0;
    double p1 = xy * xy + yz * yz + xz * xz;
    double p2 = (xx - q) * (xx - q) + (yy - q) * (yy - q) + (zz - q) * (zz - q) + 2.0 * p1;
    double p = std::sqrt(p2 / 6.0);
    if (p == 0.0) {
        out[0] = out[1] = out[2] = q;
        return;
    }
    double a = (xx - q) / p, b = (yy - q) / p, c = (zz - q) / p;
    double d = xy / p, e = yz / p, f = xz / p;
    double det = a * (b * c - e * e) - d * (d * c - e * f) + f * (d * e - b * f);
    double h = det / 2.0;
    // f64::clamp keeps a NaN.
    if (h < -1.0) h = -1.0;
    if (h > 1.0) h = 1.0;
    double phi = std::acos(h) / 3.0;
    const double pi = 3.141592653589793;
    double s1 = q + 2.0 * p * std::cos(phi);
    double s3 = q + 2.0 * p * std::cos(phi + 2.0 * pi / 3.0);
    out[0] = s1;
    out[1] = 3.0 * q - s1 - s3;
    out[2] = s3;
}

// elastic_tet.rs:164-170: D alpha, each row summed from -0.0 as the Rust float sum.
void thermal_stress(const Stiffness& d, const double alpha[3], double out[3]) {
    for (int i = 0; i < 3; ++i) {
        double s = -0.0;
        for (int j = 0; j < 3; ++j) s += d.normal[i][j] * alpha[j];
        out[i] = s;
    }
}

// elastic_tet.rs:367-427 over the cells in increasing order. `part` (NULL: 1 part) and
// `singular` (NULL: none) as the arguments of the reference's loop; the singular reason of a
// peak becomes a flag. mises_out and principal_out are elastic_tet.rs:482-483.
void recover_tet10(size_t npoints, const double* xyz, size_t nel, const uint32_t* tets10,
                   const double* coef, const double* expansion, const double* dtemp,
                   const double* u, const uint32_t* part, size_t nparts, const uint8_t* singular,
                   double* stress, double* strain, double* mises_out, double* principal_out,
                   RecoveryPeak* peaks) {
    vector<uint32_t> count(npoints, 0);
    for (size_t i = 0; i < 6 * npoints; ++i) stress[i] = strain[i] = 0.0;
    const double inf = std::numeric_limits<double>::infinity();
    vector<bool> has_regular(nparts, false);
    for (size_t p = 0; peaks && p < nparts; ++p) {
        peaks[p] = RecoveryPeak{};
        peaks[p].mises = -inf;
        peaks[p].element = -1;
        peaks[p].regular_mises = -inf;
        peaks[p].regular_element = -1;
    }
    for (size_t e = 0; e < nel; ++e) {
        const uint32_t* nodes = tets10 + 10 * e;
        Vec3 p[4], g[4];
        for (int k = 0; k < 4; ++k)
            for (int dd = 0; dd < 3; ++dd) p[k][dd] = xyz[3 * (size_t)nodes[k] + dd];
        double volume;
        tet_gradients(p, g, &volume);
        Stiffness d = isotropic_stiffness(coef[2 * e], coef[2 * e + 1]);
        double alpha[3] = {0.0, 0.0, 0.0};
        if (expansion)
            for (int k = 0; k < 3; ++k) alpha[k] = expansion[3 * e + k];
        double thermal[3];
        thermal_stress(d, alpha, thermal);
        double ue[30], te[4];
        for (int r = 0; r < 30; ++r) ue[r] = u[3 * (size_t)nodes[r / 3] + r % 3];
        for (int c = 0; c < 4; ++c) te[c] = dtemp ? dtemp[nodes[c]] : 0.0;
        bool near = false;
        if (singular)
            for (int c = 0; c < 4; ++c) near = near || singular[nodes[c]];
        size_t pt = part ? part[e] : 0;
        for (int c = 0; c < 10; ++c) {
            double l[4], eng[6], sig0[6], sig[6], eps[6];
            node_coordinates(c, l);
            tet10_strain_stress(g, d, thermal, l, ue, te, eng, sig0);
            tensor_strain(eng, eps);
            reorder_stress(sig0, sig);
            size_t node = nodes[c];
            for (int i = 0; i < 6; ++i) {
                stress[6 * node + i] += sig[i];
                strain[6 * node + i] += eps[i];
            }
            count[node] += 1;
            if (!peaks) continue;
            double vm = mises(sig);
            RecoveryPeak& pk = peaks[pt];
            bool why = (singular && singular[node]) || near;
            if (vm > pk.mises) {
                pk.mises = vm;
                pk.element = (int64_t)e;
                pk.local = c;
                pk.point = (uint32_t)node;
                pk.singular = why ? 1 : 0;
            }
            if (!why && (!has_regular[pt] || vm > pk.regular_mises)) {
                has_regular[pt] = true;
                pk.regular_mises = vm;
                pk.regular_element = (int64_t)e;
                pk.regular_local = c;
                pk.regular_point = (uint32_t)node;
            }
        }
    }
    for (size_t i = 0; i < npoints; ++i) {
        double c = (double)std::max<uint32_t>(count[i], 1u);
        for (int j = 0; j < 6; ++j) {
            stress[6 * i + j] /= c;
            strain[6 * i + j] /= c;
        }
        if (mises_out) mises_out[i] = mises(stress + 6 * i);
        if (principal_out) principal(stress + 6 * i, principal_out + 3 * i);
    }
}

// tet10.rs:51-60: the 10 quadratic functions at the volume coordinates l.
void tet10_shape(const double l[4], double n[10]) {
    for (int i = 0; i < 4; ++i) n[i] = l[i] * (2.0 * l[i] - 1.0);
    for (int k = 0; k < 6; ++k) n[4 + k] = 4.0 * l[EDGES[k][0]] * l[EDGES[k][1]];
}

// elastic_tet.rs:428-467 with cells_at (elastic_tet.rs:538-553): for each probe, the cells
// whose volume coordinates of the point are all >= -1e-9, in increasing order, each with the
// share 1 / hits of the displacement (the 10 functions), the stress (Tet10::strain_stress) and
// the temperature (the 4 corners; `temperature` NULL: 0) at the point; then the von Mises
// stress of the mean stress. Returns the first probe in no cell, or -1.
long probes_tet10(const double* xyz, size_t nel, const uint32_t* tets10, const double* coef,
                  const double* expansion, const double* dtemp, const double* temperature,
                  const double* u, size_t nprobes, const double* points, double* displacement,
                  double* stress, double* mises_out, double* temp_out, int64_t* hits_out) {
    for (size_t q = 0; q < nprobes; ++q) {
        const double* x = points + 3 * q;
        vector<std::pair<size_t, std::array<double, 4>>> hits;
        for (size_t e = 0; e < nel; ++e) {
            const uint32_t* nodes = tets10 + 10 * e;
            Vec3 p[4], g[4];
            for (int k = 0; k < 4; ++k)
                for (int dd = 0; dd < 3; ++dd) p[k][dd] = xyz[3 * (size_t)nodes[k] + dd];
            double volume;
            tet_gradients(p, g, &volume);
            std::array<double, 4> l{};
            for (int i = 1; i < 4; ++i) {
                double sum = -0.0;
                for (int dd = 0; dd < 3; ++dd) sum += g[i][dd] * (x[dd] - p[0][dd]);
                l[i] = sum;
            }
            l[0] = 1.0 - l[1] - l[2] - l[3];
            bool inside = true;
            for (int k = 0; k < 4; ++k) inside = inside && l[k] >= -1e-9;
            if (inside) hits.push_back({e, l});
        }
        if (hits_out) hits_out[q] = (int64_t)hits.size();
        if (hits.empty()) return (long)q;
        const double share = 1.0 / (double)hits.size();
        double dsp[3] = {0.0, 0.0, 0.0}, sg[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0}, tv = 0.0;
        for (const auto& h : hits) {
            const size_t e = h.first;
            const double* l = h.second.data();
            const uint32_t* nodes = tets10 + 10 * e;
            double w[10];
            tet10_shape(l, w);
            for (int c = 0; c < 10; ++c)
                for (int a = 0; a < 3; ++a) dsp[a] += share * w[c] * u[3 * (size_t)nodes[c] + a];
            Vec3 p[4], g[4];
            for (int k = 0; k < 4; ++k)
                for (int dd = 0; dd < 3; ++dd) p[k][dd] = xyz[3 * (size_t)nodes[k] + dd];
            double volume;
            tet_gradients(p, g, &volume);
            Stiffness d = isotropic_stiffness(coef[2 * e], coef[2 * e + 1]);
            double alpha[3] = {0.0, 0.0, 0.0};
            if (expansion)
                for (int k = 0; k < 3; ++k) alpha[k] = expansion[3 * e + k];
            double thermal[3];
            thermal_stress(d, alpha, thermal);
            double ue[30], te[4], eng[6], sig0[6], sig[6];
            for (int r = 0; r < 30; ++r) ue[r] = u[3 * (size_t)nodes[r / 3] + r % 3];
            for (int c = 0; c < 4; ++c) te[c] = dtemp ? dtemp[nodes[c]] : 0.0;
            tet10_strain_stress(g, d, thermal, l, ue, te, eng, sig0);
            reorder_stress(sig0, sig);
            for (int i = 0; i < 6; ++i) sg[i] += share * sig[i];
            if (temperature) {
                double sum = -0.0;
                for (int c = 0; c < 4; ++c) sum += l[c] * temperature[nodes[c]];
                tv += share * sum;
            }
        }
        for (int a = 0; a < 3; ++a) displacement[3 * q + a] = dsp[a];
        for (int i = 0; i < 6; ++i) stress[6 * q + i] = sg[i];
        mises_out[q] = mises(sg);
        temp_out[q] = tv;
    }
    return -1;
}

// elastic.rs:615-660 (the box grid): the strain and the stress at the 8 corners of each cell
// (Hex::strain_stress, hex.rs:311-335, at xi = -1 or 1 per axis), their mean at each point and
// the peaks of each part, over the cells in increasing order; `coef` holds the 9 orthotropic
// constants of each cell, `expansion` (NULL: 0) its 3 expansion coefficients. mises_out and
// principal_out are elastic.rs:709-710.
void recover_hex8(size_t npoints, const double* xyz, size_t nel, const uint32_t* hexes,
                  const double* coef, const double* expansion, const double* dtemp,
                  const double* u, const uint32_t* part, size_t nparts, const uint8_t* singular,
                  double* stress, double* strain, double* mises_out, double* principal_out,
                  RecoveryPeak* peaks) {
    static const int BITS[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                                   {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
    vector<uint32_t> count(npoints, 0);
    for (size_t i = 0; i < 6 * npoints; ++i) stress[i] = strain[i] = 0.0;
    const double inf = std::numeric_limits<double>::infinity();
    vector<bool> has_regular(nparts, false);
    for (size_t p = 0; peaks && p < nparts; ++p) {
        peaks[p] = RecoveryPeak{};
        peaks[p].mises = -inf;
        peaks[p].element = -1;
        peaks[p].regular_mises = -inf;
        peaks[p].regular_element = -1;
    }
    HexElement h;
    for (size_t e = 0; e < nel; ++e) {
        const uint32_t* nodes = hexes + 8 * e;
        double size[3], alpha[3] = {0.0, 0.0, 0.0};
        for (int d = 0; d < 3; ++d) {
            size[d] = xyz[3 * (size_t)nodes[6] + d] - xyz[3 * (size_t)nodes[0] + d];
            if (expansion) alpha[d] = expansion[3 * e + d];
        }
        const double* c9 = coef + 9 * e;
        hex8_element(size, orthotropic_stiffness(c9, c9 + 3, c9 + 6), alpha, &h);
        double ue[24], te[8];
        for (int r = 0; r < 24; ++r) ue[r] = u[3 * (size_t)nodes[r / 3] + r % 3];
        for (int c = 0; c < 8; ++c) te[c] = dtemp ? dtemp[nodes[c]] : 0.0;
        bool near = false;
        if (singular)
            for (int c = 0; c < 8; ++c) near = near || singular[nodes[c]];
        size_t pt = part ? part[e] : 0;
        for (int c = 0; c < 8; ++c) {
            double xi[3], eng[6], sig0[6], sig[6], eps[6];
            for (int d = 0; d < 3; ++d) xi[d] = BITS[c][d] == 1 ? 1.0 : -1.0;
            hex8_strain_stress(h, xi, ue, te, eng, sig0);
            tensor_strain(eng, eps);
            reorder_stress(sig0, sig);
            size_t node = nodes[c];
            for (int i = 0; i < 6; ++i) {
                stress[6 * node + i] += sig[i];
                strain[6 * node + i] += eps[i];
            }
            count[node] += 1;
            if (!peaks) continue;
            double vm = mises(sig);
            RecoveryPeak& pk = peaks[pt];
            bool why = (singular && singular[node]) || near;
            if (vm > pk.mises) {
                pk.mises = vm;
                pk.element = (int64_t)e;
                pk.local = c;
                pk.point = (uint32_t)node;
                pk.singular = why ? 1 : 0;
            }
            if (!why && (!has_regular[pt] || vm > pk.regular_mises)) {
                has_regular[pt] = true;
                pk.regular_mises = vm;
                pk.regular_element = (int64_t)e;
                pk.regular_local = c;
                pk.regular_point = (uint32_t)node;
            }
        }
    }
    for (size_t i = 0; i < npoints; ++i) {
        double c = (double)std::max<uint32_t>(count[i], 1u);
        for (int j = 0; j < 6; ++j) {
            stress[6 * i + j] /= c;
            strain[6 * i + j] /= c;
        }
        if (mises_out) mises_out[i] = mises(stress + 6 * i);
        if (principal_out) principal(stress + 6 * i, principal_out + 3 * i);
    }
}

}  // namespace orc
