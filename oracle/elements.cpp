// Oracle (test infrastructure): the element kernels of the path. Restates
// crates/fem/src/heat.rs:972-1002, 1219-1244, crates/fem/src/hex.rs:58-114 and
// crates/fem/src/tet10.rs:38-120, 232-272. The 4-node elasticity tetrahedron is this
// project's own (the reference solves elasticity on tets only with 10 nodes).
#include <algorithm>
#include <cmath>
#include <map>
#include <unordered_map>

#include "oracle.hpp"

namespace orc {

// heat.rs:983-1002
void tet_gradients(const Vec3 p[4], Vec3 g[4], double* volume) {
    double e[3][3];
    for (int k = 0; k < 3; ++k)
        for (int d = 0; d < 3; ++d) e[k][d] = p[k + 1][d] - p[0][d];
    auto cross = [](const double* a, const double* b, double* c) {
        c[0] = a[1] * b[2] - a[2] * b[1];
        c[1] = a[2] * b[0] - a[0] * b[2];
        c[2] = a[0] * b[1] - a[1] * b[0];
    };
    double det = e[0][0] * (e[1][1] * e[2][2] - e[1][2] * e[2][1]) -
                 e[0][1] * (e[1][0] * e[2][2] - e[1][2] * e[2][0]) +
                 e[0][2] * (e[1][0] * e[2][1] - e[1][1] * e[2][0]);
    double rows[3][3];
    cross(e[1], e[2], rows[0]);
    cross(e[2], e[0], rows[1]);
    cross(e[0], e[1], rows[2]);
    for (int k = 0; k < 3; ++k)
        for (int d = 0; d < 3; ++d) g[k + 1][d] = rows[k][d] / det;
    for (int d = 0; d < 3; ++d) g[0][d] = -(g[1][d] + g[2][d] + g[3][d]);
    *volume = det / 6.0;
}

// heat.rs:972-981. The Rust float sum starts from -0.0, the exact additive identity, so it
// equals ((t0 + t1) + t2).
void tet_conduction(const Vec3 g[4], double v, const Vec3& k, double ke[16]) {
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            double s = k[0] * g[i][0] * g[j][0];
            s = s + k[1] * g[i][1] * g[j][1];
            s = s + k[2] * g[i][2] * g[j][2];
            ke[i * 4 + j] = v * s;
        }
}

// heat.rs:1219-1244; `capacity` null is `transient = None`, else Some((capacity, dt)).
vector<double> reduced_rhs(const Csr& a, const double* load, const double* t,
                           const vector<size_t>& free, const double* capacity, double dt) {
    vector<double> out(free.size());
    for (size_t k = 0; k < free.size(); ++k) {
        size_t i = free[k];
        double r = load[i];
        if (capacity) r += capacity[i] / dt * t[i];
        for (size_t e = a.ptr[i]; e < a.ptr[i + 1]; ++e) {
            size_t j = a.idx[e];
            if (!std::binary_search(free.begin(), free.end(), j)) r -= a.val[e] * t[j];
        }
        out[k] = r;
    }
    return out;
}

// hex.rs:69-114
Stiffness orthotropic_stiffness(const double e[3], const double nu[3], const double g[3]) {
    for (int i = 0; i < 3; ++i)
        if (!(std::isfinite(e[i]) && e[i] > 0.0 && std::isfinite(g[i]) && g[i] > 0.0) ||
            !std::isfinite(nu[i]))
            throw Error("the moduli must be above 0 and the Poisson ratios finite");
    double ex = e[0], ey = e[1], ez = e[2];
    double nxy = nu[0], nxz = nu[1], nyz = nu[2];
    double s[3][3] = {{1.0 / ex, -nxy / ex, -nxz / ex},
                      {-nxy / ex, 1.0 / ey, -nyz / ey},
                      {-nxz / ex, -nyz / ey, 1.0 / ez}};
    double det = s[0][0] * (s[1][1] * s[2][2] - s[1][2] * s[2][1]) -
                 s[0][1] * (s[1][0] * s[2][2] - s[1][2] * s[2][0]) +
                 s[0][2] * (s[1][0] * s[2][1] - s[1][1] * s[2][0]);
    double minor = s[0][0] * s[1][1] - s[0][1] * s[1][0];
    if (!(minor > 0.0 && det > 1e-12 * s[0][0] * s[1][1] * s[2][2]))
        throw Error(
            "the Poisson ratios give no stable material (for an isotropic material, nu must be "
            "between -1 and 0.5)");
    Stiffness d;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
            d.normal[i][j] = (s[j1][i1] * s[j2][i2] - s[j1][i2] * s[j2][i1]) / det;
        }
    d.shear[0] = g[2];  // G_yz
    d.shear[1] = g[1];  // G_xz
    d.shear[2] = g[0];  // G_xy
    return d;
}

// hex.rs:58-64
Stiffness isotropic_stiffness(double e, double nu) {
    double ee[3] = {e, e, e}, nn[3] = {nu, nu, nu};
    double gg = e / (2.0 * (1.0 + nu));
    double g[3] = {gg, gg, gg};
    return orthotropic_stiffness(ee, nn, g);
}

// tet10.rs:41: the 2 axes of each shear strain (yz, xz, xy).
static const int SHEAR[3][2] = {{1, 2}, {0, 2}, {0, 1}};
// tet10.rs:38
static const int EDGES[6][2] = {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {1, 3}, {2, 3}};

// The (a, b) term of the B^T D B integrand of 2 node gradients: tet10.rs:101-112.
static inline double elastic_term(const double* gi, const double* gj, int a, int b,
                                  const Stiffness& d) {
    double v = gi[a] * gj[b] * d.normal[a][b];
    if (a == b) {
        for (int s = 0; s < 3; ++s) {
            int p = SHEAR[s][0], q = SHEAR[s][1];
            if (p == a)
                v += gi[q] * gj[q] * d.shear[s];
            else if (q == a)
                v += gi[p] * gj[p] * d.shear[s];
        }
    } else {
        v += gi[b] * gj[a] * d.shear[3 - a - b];
    }
    return v;
}

// tet10.rs:44-48 and 77-87: the 4-point rule of degree 2 and the gradients of the 10 functions.
void tet10_stiffness(const Vec3 g[4], double volume, const Stiffness& d, double k[900]) {
    const double A = 0.5854101966249685, B = 0.1381966011250105;
    std::fill(k, k + 900, 0.0);
    double w = volume / 4.0;
    for (int q = 0; q < 4; ++q) {
        double l[4];
        for (int c = 0; c < 4; ++c) l[c] = (c == q) ? A : B;
        double gr[10][3];
        for (int i = 0; i < 4; ++i)
            for (int dd = 0; dd < 3; ++dd) gr[i][dd] = (4.0 * l[i] - 1.0) * g[i][dd];
        for (int e = 0; e < 6; ++e) {
            int i = EDGES[e][0], j = EDGES[e][1];
            for (int dd = 0; dd < 3; ++dd)
                gr[4 + e][dd] = 4.0 * (l[i] * g[j][dd] + l[j] * g[i][dd]);
        }
        for (int i = 0; i < 10; ++i)
            for (int j = 0; j < 10; ++j)
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < 3; ++b)
                        k[(3 * i + a) * 30 + 3 * j + b] += w * elastic_term(gr[i], gr[j], a, b, d);
    }
}

// The 4-node tetrahedron: constant gradients, 1 point of weight V, same layout as tet10.rs:113.
void tet4_stiffness(const Vec3 g[4], double volume, const Stiffness& d, double k[144]) {
    std::fill(k, k + 144, 0.0);
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j)
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b)
                    k[(3 * i + a) * 12 + 3 * j + b] += volume * elastic_term(g[i].data(), g[j].data(), a, b, d);
}

// tet10.rs:244-272: edge points numbered in the order of first sight over (tetrahedron,
// EDGES order), keyed by the sorted corner pair.
Quadratic quadratic(const vector<Vec3>& points, const vector<array<uint32_t, 4>>& tets) {
    Quadratic q;
    q.corners = points.size();
    std::unordered_map<uint64_t, uint32_t> of;
    of.reserve(tets.size() * 2);
    q.tets.reserve(tets.size());
    for (const auto& tet : tets) {
        array<uint32_t, 10> t{};
        for (int c = 0; c < 4; ++c) t[c] = tet[c];
        for (int k = 0; k < 6; ++k) {
            uint32_t a = std::min(tet[EDGES[k][0]], tet[EDGES[k][1]]);
            uint32_t b = std::max(tet[EDGES[k][0]], tet[EDGES[k][1]]);
            uint64_t key = ((uint64_t)a << 32) | b;
            auto it = of.find(key);
            if (it == of.end()) {
                q.edges.push_back({a, b});
                uint32_t id = (uint32_t)(q.corners + q.edges.size() - 1);
                of.emplace(key, id);
                t[4 + k] = id;
            } else {
                t[4 + k] = it->second;
            }
        }
        q.tets.push_back(t);
    }
    q.points = points;
    for (const auto& e : q.edges) {
        const Vec3 &p = points[e[0]], &r = points[e[1]];
        q.points.push_back({0.5 * (p[0] + r[0]), 0.5 * (p[1] + r[1]), 0.5 * (p[2] + r[2])});
    }
    return q;
}

// The priority of an element in the colouring: the "lowbias32" integer hash of C. Wellons
// (2018), a bijection of 32-bit words.
uint32_t colour_priority(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    x *= 0x846ca68bU;
    x ^= x >> 16;
    return x;
}

// Jones-Plassmann colouring: M. T. Jones and P. E. Plassmann, A parallel graph coloring
// heuristic, SIAM J. Sci. Comput. 14 (1993) 654-669. In each round an uncoloured element whose
// (priority, index) is above that of each uncoloured element it shares a node with takes the
// smallest colour that no coloured element it shares a node with has. Elements that share a
// node get different colours, so the scatter of 1 colour has no write conflicts.
vector<uint32_t> colour_elements(size_t n, const uint32_t* elements, size_t nel, int m,
                                 int* ncolours) {
    const uint32_t UNSET = UINT32_MAX;
    vector<size_t> count(n + 1, 0);
    for (size_t e = 0; e < nel; ++e)
        for (int a = 0; a < m; ++a) count[elements[e * m + a] + 1] += 1;
    for (size_t i = 0; i < n; ++i) count[i + 1] += count[i];
    vector<uint32_t> of_node(count[n]);
    vector<size_t> next(count);
    for (size_t k = 0; k < nel; ++k)
        for (int a = 0; a < m; ++a) of_node[next[elements[k * m + a]]++] = (uint32_t)k;
    vector<uint32_t> colour(nel, UNSET);
    vector<char> selected(nel, 0);
    size_t left = nel;
    int most = 0;
    while (left > 0) {
        for (size_t e = 0; e < nel; ++e) {
            selected[e] = 0;
            if (colour[e] != UNSET) continue;
            uint64_t me = ((uint64_t)colour_priority((uint32_t)e) << 32) | (uint32_t)e;
            bool top = true;
            for (int a = 0; a < m && top; ++a) {
                uint32_t v = elements[e * m + a];
                for (size_t t = count[v]; t < count[v + 1]; ++t) {
                    uint32_t f = of_node[t];
                    if (f == e || colour[f] != UNSET) continue;
                    uint64_t other = ((uint64_t)colour_priority(f) << 32) | f;
                    if (other > me) {
                        top = false;
                        break;
                    }
                }
            }
            selected[e] = top;
        }
        for (size_t e = 0; e < nel; ++e) {
            if (!selected[e]) continue;
            uint64_t used[4] = {0, 0, 0, 0};
            for (int a = 0; a < m; ++a) {
                uint32_t v = elements[e * m + a];
                for (size_t t = count[v]; t < count[v + 1]; ++t) {
                    uint32_t c = colour[of_node[t]];
                    if (c != UNSET && c < 256) used[c >> 6] |= 1ull << (c & 63);
                }
            }
            uint32_t c = 0;
            while (c < 256 && (used[c >> 6] >> (c & 63) & 1)) ++c;
            if (c >= 256) throw Error("the elements need more than 256 colours");
            colour[e] = c;
            most = std::max(most, (int)c + 1);
            --left;
        }
    }
    *ncolours = most;
    return colour;
}

// heat.rs:691-696
void add_capacity(Csr* a, const double* capacity, double dt) {
    for (size_t i = 0; i < a->n; ++i) {
        size_t d;
        if (!a->find(i, i, &d)) throw Error("a diagonal");
        a->val[d] += capacity[i] / dt;
    }
}

// heat.rs:535-547 with rad = 0 (the transient path of heat.rs:717-733 passes no radiation).
void transient_energy(size_t n, const double* kt, const double* rate, const double* load,
                      const uint8_t* fixed, double out[3]) {
    double stored = 0.0, fix = 0.0, gross = 0.0;
    for (size_t i = 0; i < n; ++i) {
        stored += rate[i];
        gross += std::fabs(rate[i]);
        gross += 0.0;  // |rad[i]|
        if (fixed[i]) {
            double q = kt[i] + rate[i] - load[i] - 0.0;
            fix += q;
            gross += std::fabs(q);
        }
    }
    out[0] = stored;
    out[1] = fix;
    out[2] = gross;
}

// heat.rs:1246-1273: the 8 x 8 conduction matrix of a box cell of sides s, VTK corner order.
void hex_conduction(const double s[3], const double k[3], double ke[64]) {
    static const int BITS[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                                   {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
    for (int p = 0; p < 8; ++p)
        for (int q = 0; q < 8; ++q) {
            double v = 0.0;
            for (int d = 0; d < 3; ++d) {
                double term = k[d];
                for (int e = 0; e < 3; ++e) {
                    bool same = BITS[p][e] == BITS[q][e];
                    term *= e == d ? (same ? 1.0 / s[e] : -1.0 / s[e])
                                   : (same ? s[e] / 3.0 : s[e] / 6.0);
                }
                v += term;
            }
            ke[p * 8 + q] = v;
        }
}

// hex.rs:146-160: the gradients of the 8 corner functions and the 3 mode functions at the local
// point xi of a box of sides `size`.
static void hex_gradients(const double size[3], const double xi[3], double g[11][3]) {
    static const int BITS[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                                   {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
    for (int i = 0; i < 11; ++i)
        for (int d = 0; d < 3; ++d) g[i][d] = 0.0;
    for (int n = 0; n < 8; ++n) {
        double s[3], f[3];
        for (int d = 0; d < 3; ++d) {
            s[d] = BITS[n][d] == 1 ? 1.0 : -1.0;
            f[d] = 0.5 * (1.0 + s[d] * xi[d]);
        }
        for (int d = 0; d < 3; ++d) g[n][d] = s[d] / size[d] * f[(d + 1) % 3] * f[(d + 2) % 3];
    }
    for (int d = 0; d < 3; ++d) g[8 + d][d] = -4.0 * xi[d] / size[d];
}

// hex.rs:164-178: the values of the 8 corner functions at xi (a product from 1.0).
static void hex_shape(const double xi[3], double n[8]) {
    static const int BITS[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                                   {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
    for (int c = 0; c < 8; ++c) {
        double v = 1.0;
        for (int d = 0; d < 3; ++d) v *= BITS[c][d] == 1 ? 0.5 * (1.0 + xi[d]) : 0.5 * (1.0 - xi[d]);
        n[c] = v;
    }
}

// hex.rs:218-309: Hex::new. The 33 x 33 stiffness and the 33 x 8 thermal load of the 8 corner
// and 3 mode functions over the 2-point Gauss rule, then the 9 modes condensed with the Cholesky
// factor of their block (hex.rs:355-389).
void hex8_element(const double size[3], const Stiffness& d, const double alpha[3], HexElement* h) {
    static const int BITS[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                                   {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
    for (int d3 = 0; d3 < 3; ++d3) h->size[d3] = size[d3];
    h->d = d;
    for (int i = 0; i < 3; ++i) {  // the Rust float sum starts from -0.0
        double s = -0.0;
        for (int j = 0; j < 3; ++j) s += d.normal[i][j] * alpha[j];
        h->thermal[i] = s;
    }
    double k[33][33], l[33][8];
    for (int i = 0; i < 33; ++i) {
        for (int j = 0; j < 33; ++j) k[i][j] = 0.0;
        for (int c = 0; c < 8; ++c) l[i][c] = 0.0;
    }
    const double jac = size[0] * size[1] * size[2] / 8.0;
    const double p = 1.0 / std::sqrt(3.0);
    for (int gp = 0; gp < 8; ++gp) {
        double xi[3], g[11][3], n[8];
        for (int e = 0; e < 3; ++e) xi[e] = BITS[gp][e] == 1 ? p : -p;
        hex_gradients(size, xi, g);
        hex_shape(xi, n);
        for (int i = 0; i < 11; ++i) {
            for (int j = 0; j < 11; ++j)
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < 3; ++b)
                        k[3 * i + a][3 * j + b] += jac * elastic_term(g[i], g[j], a, b, d);
            for (int a = 0; a < 3; ++a)
                for (int c = 0; c < 8; ++c) l[3 * i + a][c] += jac * g[i][a] * h->thermal[a] * n[c];
        }
    }
    double ch[9][9] = {};
    for (int j = 0; j < 9; ++j) {  // cholesky9
        double dd = k[24 + j][24 + j];
        for (int c = 0; c < j; ++c) dd -= ch[j][c] * ch[j][c];
        dd = std::sqrt(dd);
        ch[j][j] = dd;
        for (int i = j + 1; i < 9; ++i) {
            double v = k[24 + i][24 + j];
            for (int c = 0; c < j; ++c) v -= ch[i][c] * ch[j][c];
            ch[i][j] = v / dd;
        }
    }
    auto solve9 = [&](double b[9]) {
        for (int i = 0; i < 9; ++i) {
            for (int q = 0; q < i; ++q) b[i] -= ch[i][q] * b[q];
            b[i] /= ch[i][i];
        }
        for (int i = 8; i >= 0; --i) {
            for (int q = i + 1; q < 9; ++q) b[i] -= ch[q][i] * b[q];
            b[i] /= ch[i][i];
        }
    };
    for (int c = 0; c < 24; ++c) {
        double b[9];
        for (int i = 0; i < 9; ++i) b[i] = k[24 + i][c];
        solve9(b);
        for (int i = 0; i < 9; ++i) h->mode_u[i * 24 + c] = b[i];
    }
    for (int c = 0; c < 8; ++c) {
        double b[9];
        for (int i = 0; i < 9; ++i) b[i] = l[24 + i][c];
        solve9(b);
        for (int i = 0; i < 9; ++i) h->mode_t[i * 8 + c] = b[i];
    }
    for (int r = 0; r < 24; ++r) {
        for (int c = 0; c < 24; ++c) {
            double v = k[r][c];
            for (int i = 0; i < 9; ++i) v -= k[r][24 + i] * h->mode_u[i * 24 + c];
            h->k[r * 24 + c] = v;
        }
        for (int c = 0; c < 8; ++c) {
            double v = l[r][c];
            for (int i = 0; i < 9; ++i) v -= k[r][24 + i] * h->mode_t[i * 8 + c];
            h->load[r * 8 + c] = v;
        }
    }
}

// hex.rs:337-353: the consistent mass of the 24 corner unknowns, rho times the product of the
// 1D masses (a / 3 at the same end, a / 6 across).
void hex8_mass(const double size[3], double density, double m[576]) {
    static const int BITS[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                                   {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
    for (int k = 0; k < 576; ++k) m[k] = 0.0;
    for (int i = 0; i < 8; ++i)
        for (int j = 0; j < 8; ++j) {
            double v = 1.0;
            for (int d = 0; d < 3; ++d)
                v *= BITS[i][d] == BITS[j][d] ? size[d] / 3.0 : size[d] / 6.0;
            for (int a = 0; a < 3; ++a) m[(3 * i + a) * 24 + 3 * j + a] = density * v;
        }
}

void hex8_stiffness(const double size[3], const Stiffness& d, double kc[576]) {
    const double zero[3] = {0.0, 0.0, 0.0};
    HexElement h;
    hex8_element(size, d, zero, &h);
    for (int i = 0; i < 576; ++i) kc[i] = h.k[i];
}

// hex.rs:311-335: the engineering strain and the stress (xx, yy, zz, yz, xz, xy) at the local
// point xi from the corner displacements u and the corner temperature changes t.
void hex8_strain_stress(const HexElement& h, const double xi[3], const double u[24],
                        const double t[8], double e[6], double s[6]) {
    static const int SH[3][2] = {{1, 2}, {0, 2}, {0, 1}};
    double all[11][3];
    for (int n = 0; n < 8; ++n)
        for (int a = 0; a < 3; ++a) all[n][a] = u[3 * n + a];
    for (int i = 0; i < 9; ++i) {
        double a = 0.0;
        for (int c = 0; c < 8; ++c) a += h.mode_t[i * 8 + c] * t[c];
        for (int c = 0; c < 24; ++c) a -= h.mode_u[i * 24 + c] * u[c];
        all[8 + i / 3][i % 3] = a;
    }
    double g[11][3], n[8];
    hex_gradients(h.size, xi, g);
    for (int a = 0; a < 6; ++a) e[a] = 0.0;
    for (int i = 0; i < 11; ++i) {
        for (int a = 0; a < 3; ++a) e[a] += g[i][a] * all[i][a];
        for (int q = 0; q < 3; ++q) {
            const int a = SH[q][0], b = SH[q][1];
            e[3 + q] += g[i][a] * all[i][b] + g[i][b] * all[i][a];
        }
    }
    hex_shape(xi, n);
    double dt = -0.0;
    for (int c = 0; c < 8; ++c) dt += n[c] * t[c];
    for (int a = 0; a < 3; ++a)  // hex.rs:128-139
        s[a] = h.d.normal[a][0] * e[0] + h.d.normal[a][1] * e[1] + h.d.normal[a][2] * e[2];
    for (int q = 0; q < 3; ++q) s[3 + q] = h.d.shear[q] * e[3 + q];
    for (int a = 0; a < 3; ++a) s[a] -= h.thermal[a] * dt;
}

// elastic.rs:386-405 (the force part): over the cells in increasing order, each unknown of each
// cell gets f = sum_c load[r][c] T_c (from 0.0), plus (its acceleration term, density g_d +
// body_d, given per cell as `accel`) times the volume / 8. `force` (3 per point) is zeroed first.
void hex_loads(size_t npoints, const double* xyz, size_t nel, const uint32_t* hexes,
               const double* coef, const double* expansion, const double* accel,
               const double* dtemp, double* force) {
    for (size_t i = 0; i < 3 * npoints; ++i) force[i] = 0.0;
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
        double t[8];
        for (int c = 0; c < 8; ++c) t[c] = dtemp ? dtemp[nodes[c]] : 0.0;
        const double volume = size[0] * size[1] * size[2];
        for (int r = 0; r < 24; ++r) {
            double f = 0.0;
            for (int c = 0; c < 8; ++c) f += h.load[r * 8 + c] * t[c];
            const int d = r % 3;
            f += (accel ? accel[3 * e + d] : 0.0) * volume / 8.0;
            force[3 * (size_t)nodes[r / 3] + d] += f;
        }
    }
}

}  // namespace orc

