// CPU oracle: a C++17 restatement of the fh-fem iterative solve path of femahoy (crates/fem).
//
// TEST INFRASTRUCTURE ONLY. This library is the checker of the CUDA path: only the tests, the
// smoke check and the CPU-baseline leg of the benchmark load it. The product (libfemgpu.so)
// never links, calls or falls back to it.
//
// Every function cites the reference file:line it restates (paths inside the femahoy project).
// Floating-point expressions keep the reference's evaluation order, and the build uses
// -ffp-contract=off, so that element matrices and assembled values are bit-identical with
// the Rust code (which never fuses a multiply and an add).
#pragma once
#include <cstddef>
#include <cstdint>
#include <functional>
#include <stdexcept>
#include <string>
#include <vector>
#include <array>

namespace orc {

using std::size_t;
using std::vector;
using std::array;

constexpr size_t NONE = SIZE_MAX;  // symbolic.rs:14

// A failure with the reference's error text (the Rust `Err(String)`).
struct Error : std::runtime_error {
    explicit Error(const std::string& s) : std::runtime_error(s) {}
};

// Rust's LowerExp text of v, as the reference's format! strings write it: digits >= 0 is
// "{:.digits$e}" (multigrid.rs:730-732 uses 2), digits < 0 is "{:e}", the shortest digits that
// read back to v (cholesky.rs:92-97). The exponent is a bare integer (1.23e-5, 2.5e0).
std::string rust_lower_exp(double v, int digits);

// ---------------------------------------------------------------- sparse.rs
// sparse.rs:12-17: square CSR with both triangles, sorted columns per row.
// Host threads of the parallel parts of the restatement: the matrix product and the PCG dot
// products (the reference runs on 1 thread; 1 is the default and gives its arithmetic).
void set_threads(int n);
int threads();

struct Csr {
    size_t n = 0;
    vector<size_t> ptr;
    vector<uint32_t> idx;
    vector<double> val;
    // sparse.rs:68-71
    bool find(size_t i, size_t j, size_t* at) const;
    // sparse.rs:75-86
    void add_element(const uint32_t* nodes, int m, const double* ke);
    // sparse.rs:89-93
    vector<double> diagonal() const;
    // sparse.rs:96-105
    void mul(const double* x, double* y) const;
    // sparse.rs:108-135
    Csr submatrix(const vector<size_t>& keep) const;
};
// sparse.rs:22-65: elements are `nel` runs of `m` nodes.
Csr pattern(size_t n, const uint32_t* elements, size_t nel, int m);
// The same for elements of different sizes: element k is nodes[start[k] .. start[k + 1]].
Csr pattern_lists(size_t n, const vector<uint32_t>& nodes, const vector<size_t>& start);

// sparse.rs:202-208
struct Rect {
    size_t rows = 0, cols = 0;
    vector<size_t> ptr;
    vector<uint32_t> idx;
    vector<double> val;
    void mul(const double* x, double* y) const;            // sparse.rs:212-220
    void mul_transpose(const double* x, double* y) const;  // sparse.rs:223-230
    Csr galerkin(const Csr& a) const;                       // sparse.rs:233-292
};

// ---------------------------------------------------------------- elements
using Vec3 = array<double, 3>;
// heat.rs:983-1002
void tet_gradients(const Vec3 p[4], Vec3 g[4], double* volume);
// heat.rs:972-981
void tet_conduction(const Vec3 g[4], double v, const Vec3& k, double ke[16]);
// heat.rs:1219-1244 (steady form: no transient term)
vector<double> reduced_rhs(const Csr& a, const double* load, const double* t,
                           const vector<size_t>& free, const double* capacity = nullptr,
                           double dt = 0.0);
// heat.rs:691-696: a_full = K with capacity / dt added to each diagonal entry.
void add_capacity(Csr* a, const double* capacity, double dt);
// heat.rs:535-547 for a transient step with no radiation: out = {stored, fixed, the sum of
// |rate| and |q| over the points}, each summed in point order.
void transient_energy(size_t n, const double* kt, const double* rate, const double* load,
                      const uint8_t* fixed, double out[3]);

// hex.rs:120-124
struct Stiffness {
    double normal[3][3];
    double shear[3];  // G_yz, G_xz, G_xy
};
// hex.rs:58-64 then hex.rs:69-114
Stiffness isotropic_stiffness(double e, double nu);
Stiffness orthotropic_stiffness(const double e[3], const double nu[3], const double g[3]);

// tet10.rs:90-120: 30 x 30 row-major, unknown 3 node + component.
void tet10_stiffness(const Vec3 g[4], double volume, const Stiffness& d, double k[900]);
// The linear (4-node) elasticity tetrahedron, which the reference lacks: V B^T D B with the
// constant gradients of tet_gradients, in the index layout and term order of tet10.rs:99-113.
void tet4_stiffness(const Vec3 g[4], double volume, const Stiffness& d, double k[144]);

// tet10.rs:173-212
void tet10_mass(double volume, double density, double m[900]);
// heat.rs:1246-1273
void hex_conduction(const double s[3], const double k[3], double ke[64]);
// hex.rs:218-297, 355-389: the condensed 24 x 24 stiffness of a box cell
void hex8_stiffness(const double size[3], const Stiffness& d, double kc[576]);
// hex.rs:186-309 `Hex`: the box cell's condensed stiffness, its load of a unit temperature
// change at each corner, and the mode amplitudes a = mode_t T - mode_u u.
struct HexElement {
    double size[3];
    Stiffness d;
    double thermal[3];
    double k[576], load[192], mode_u[216], mode_t[72];
};
void hex8_element(const double size[3], const Stiffness& d, const double alpha[3], HexElement* h);
// hex.rs:337-353
void hex8_mass(const double size[3], double density, double m[576]);
// elastic.rs:386-405: the thermal and volume forces of the box cells (3 per point).
void hex_loads(size_t npoints, const double* xyz, size_t nel, const uint32_t* hexes,
               const double* coef, const double* expansion, const double* accel,
               const double* dtemp, double* force);
// hex.rs:311-335
void hex8_strain_stress(const HexElement& h, const double xi[3], const double u[24],
                        const double t[8], double e[6], double s[6]);

// eigen.rs:183-269 and 274-331: the dense generalized and standard symmetric eigenproblems.
// Returns false with `err` set when M is not positive definite.
bool dense_generalized(const double* k, const double* m, int n, double* values, double* q,
                       std::string* err);
void dense_jacobi(double* a, int n, double* values, double* v);

// tet10.rs:232-272
struct Quadratic {
    vector<Vec3> points;
    size_t corners = 0;
    vector<array<uint32_t, 2>> edges;
    vector<array<uint32_t, 10>> tets;
};
Quadratic quadratic(const vector<Vec3>& points, const vector<array<uint32_t, 4>>& tets);

// Element colouring (not in the reference, whose assembly is sequential; sparse.rs:75):
// Jones-Plassmann with a fixed integer hash as the priority and first-fit colours. The CUDA
// colouring runs the same rounds, so both give the same colour for each element.
uint32_t colour_priority(uint32_t e);
vector<uint32_t> colour_elements(size_t n, const uint32_t* elements, size_t nel, int m,
                                 int* ncolours);

// ---------------------------------------------------------------- post-solve recovery
// elastic_tet.rs:367-427: the peak von Mises stress of a part over the 10 points of its cells,
// and the same over the points that are not singular (the reference's `Peak`). A part with no
// cells keeps mises -inf and element -1; regular_element -1 is the reference's `None`.
struct RecoveryPeak {
    double mises;
    int64_t element;
    int32_t local;
    uint32_t point;
    int32_t singular;
    int32_t pad;
    double regular_mises;
    int64_t regular_element;
    int32_t regular_local;
    uint32_t regular_point;
};
// elastic_tet.rs:367-427 and 482-483 for isotropic materials (E, nu per cell as the assembly):
// the mean strain (tensor components) and stress (xx, yy, zz, xy, yz, xz) at each point, the
// von Mises and principal stresses of the mean, and the peaks of each part.
void recover_tet10(size_t npoints, const double* xyz, size_t nel, const uint32_t* tets10,
                   const double* coef, const double* expansion, const double* dtemp,
                   const double* u, const uint32_t* part, size_t nparts, const uint8_t* singular,
                   double* stress, double* strain, double* mises_out, double* principal_out,
                   RecoveryPeak* peaks);
// elastic.rs:615-660 and 709-710 for box cells (8 corners in VTK order, 9 orthotropic constants
// per cell): as recover_tet10 over the 8 corners of each cell.
void recover_hex8(size_t npoints, const double* xyz, size_t nel, const uint32_t* hexes,
                  const double* coef, const double* expansion, const double* dtemp,
                  const double* u, const uint32_t* part, size_t nparts, const uint8_t* singular,
                  double* stress, double* strain, double* mises_out, double* principal_out,
                  RecoveryPeak* peaks);
// elastic.rs:977-1002
double mises(const double s[6]);
void principal(const double s[6], double out[3]);

// ---------------------------------------------------------------- order / symbolic / cholesky
// order.rs:19-179
vector<size_t> nested_dissection(const Csr& a, const vector<Vec3>& xyz);

// symbolic.rs:19-192
struct Symbolic {
    size_t n = 0;
    vector<size_t> perm, iperm, start, rows_ptr;
    vector<uint32_t> rows;
    vector<size_t> parent, children;
    size_t supernodes() const { return start.size() - 1; }
    uint64_t entries() const;  // symbolic.rs:162-170
    double flops() const;      // symbolic.rs:174-182
};
Symbolic analyse(const Csr& a, const vector<size_t>& order);

// cholesky.rs:23-167
struct Cholesky {
    Symbolic sym;
    vector<size_t> offset;
    vector<double> values;
    void solve(double* b) const;  // cholesky.rs:125-160
};
Cholesky factor(const Symbolic& sym, const Csr& a);  // cholesky.rs:44-122

// ---------------------------------------------------------------- multigrid.rs
// multigrid.rs:55-59
struct Level {
    array<vector<double>, 3> planes;
    vector<array<uint32_t, 3>> points;
    vector<uint8_t> comp;
};

// multigrid.rs:187-324
struct Lines {
    vector<uint32_t> order;
    vector<size_t> start;
    vector<uint32_t> line, place;
    size_t band = 0;
    vector<double> factor;
    static Lines make(const Level& level, int axis, const Csr& a);
    void sweep(const Csr& a, const double* b, double* x, bool forward) const;
};

// multigrid.rs:329-452
bool coarsen(const Level& fine, const Csr& a, Rect* p, Level* coarse);

// multigrid.rs:62-68 `Cells`: the lowest grid point of each cell of a displacement model and
// its 24 x 24 matrix (row-major, unknown 3 n + c for corner n in VTK order), here the class
// matrix table + 576 cls[i].
struct Cells {
    vector<array<uint32_t, 3>> origin;
    vector<uint32_t> cls;
    vector<double> table;
    const double* element(size_t i) const { return table.data() + 576 * (size_t)cls[i]; }
    bool empty() const { return origin.empty(); }
};

// multigrid.rs:458-608: the coarse matrix of a displacement from the cells, and the coarse
// cells with their matrices for the next level.
Csr by_cells(const Level& fine, const Cells& cells, const Level& coarse, Cells* next);

// multigrid.rs:73-180; with `cells` the coarse matrices come from the cells.
struct Multigrid {
    vector<Csr> a;
    vector<Rect> p;
    vector<array<Lines, 3>> lines;
    Cholesky coarse;
    static Multigrid make(const Csr& a, Level level, const Cells* cells = nullptr);
    size_t levels() const { return a.size(); }
    void apply(const double* r, double* z) const;
    void cycle(size_t l, const double* b, double* x) const;
};

// multigrid.rs:683-753
struct Convergence {
    size_t iterations;
    double residual;
};
Convergence pcg(const Csr& a, const double* b, double* x,
                const std::function<void(const double*, double*)>& precondition, double tol,
                size_t max_iter, const std::function<bool()>& cancelled);

// ---------------------------------------------------------------- pmultigrid.rs
struct PMultigrid {
    Rect p;
    vector<double> diag;
    Cholesky coarse;
    size_t coarse_unknowns = 0;
    static PMultigrid make(const Csr& a, Rect p, const vector<Vec3>& coarse);  // :46-60
    void apply(const Csr& a, const double* r, double* z) const;               // :63-98
};
// pmultigrid.rs:104-151
void prolongation(const vector<Vec3>& points, size_t corners,
                  const vector<array<uint32_t, 2>>& edges, const vector<size_t>& free, Rect* p,
                  vector<Vec3>* xyz);

// ---------------------------------------------------------------- solve.rs
constexpr size_t STEADY_DIRECT_LIMIT = 3000;    // solve.rs:18
constexpr size_t TRANSIENT_DIRECT_LIMIT = 40000;  // solve.rs:24
constexpr double PCG_TOL = 1e-10;               // solve.rs:42
constexpr size_t PCG_MAX_ITER = 500;            // solve.rs:43

enum class Method { Direct = 0, Multigrid = 1 };  // solve.rs:47-50

// solve.rs:28-39
struct Crossover {
    bool flops_rule = false;
    size_t unknowns = STEADY_DIRECT_LIMIT;
    double flops = 0.0;
    uint64_t entries = 0;
    bool flat = false;
};

// solve.rs:64-77
struct Unknowns {
    enum Kind { Grid = 0, Points = 1, Quadratic = 2 } kind = Grid;
    Level level;             // Grid
    Cells cells;             // Grid: solve.rs:97 `cells` (empty: None)
    vector<Vec3> points;     // Points, Quadratic
    Rect p;                  // Quadratic
    vector<Vec3> coarse;     // Quadratic
};

struct Stats {
    size_t iterations;
    double residual;
};

// solve.rs:58-250
struct Solver {
    enum Inner { Direct, MG, PMG } inner = Direct;
    Csr a;
    Cholesky chol;
    Multigrid mg;
    PMultigrid pmg;
    size_t max_iter = PCG_MAX_ITER;
    double tol = PCG_TOL;
    static Solver make(Csr a, Unknowns unknowns, int method /* -1 none */, Crossover crossover);
    Method method() const { return inner == Direct ? Method::Direct : Method::Multigrid; }
    Stats solve(const double* b, double* x, const std::function<bool()>& cancelled) const;
};

// elastic.rs:772-839 (reactions.cpp): r = K u - f at the fixed unknowns summed per owner
// load (3 per load), per component into total (from `applied`) and into the gross magnitude.
void reactions(const Csr& k, const double* u, const double* force, const uint8_t* fixed,
               const uint32_t* owner, size_t nloads, const double applied[3], double gross,
               double* load_force, double total[3], double* gross_out, double* imbalance);

// elastic_tet.rs:428-467 (recover.cpp): the probes of a P2 model; the first probe in no cell,
// or -1.
long probes_tet10(const double* xyz, size_t nel, const uint32_t* tets10, const double* coef,
                  const double* expansion, const double* dtemp, const double* temperature,
                  const double* u, size_t nprobes, const double* points, double* displacement,
                  double* stress, double* mises_out, double* temp_out, int64_t* hits_out);

}  // namespace orc
