// Device assembly: the interfaces of assemble.cu.
#pragma once
#include "common.cuh"

namespace femgpu {

// The elements of each node, in increasing element order: of_node[start[v] .. start[v + 1]].
struct Incidence {
    int64_t n = 0, nel = 0;
    int m = 0;
    DevBuf<int64_t> start;
    DevBuf<uint32_t> of_node;
};

// The result of an assembly: the matrix, the pattern of the nodes (elasticity) and the
// incidence it was built from.
struct Assembled {
    DevCsr matrix;
    DevCsr node;
    Incidence inc;
    int ncolours = 0;
};

void build_incidence(const uint32_t* d_el, int64_t nel, int m, int64_t n, Incidence* inc,
                     cudaStream_t s);
void build_pattern(const uint32_t* d_el, const Incidence& inc, DevCsr* out, cudaStream_t s);
int colour_elements(const uint32_t* d_el, const Incidence& inc, DevBuf<uint32_t>* colour,
                    cudaStream_t s);
void assemble(int kind, int mode, int64_t npoints, const double* d_xyz, int64_t nel,
              const uint32_t* d_el, const double* d_coef, Assembled* out, cudaStream_t s);
int64_t quadratic(int64_t ncorner, int64_t ntet, const uint32_t* d_tets, uint32_t* d_tets10,
                  uint32_t* d_edges, cudaStream_t s);
void submatrix(const DevCsr& a, const int64_t* d_keep, int64_t nkeep, DevCsr* out,
               cudaStream_t s);
void reduced_rhs(const DevCsr& a, const double* d_load, const double* d_t, const int64_t* d_free,
                 int64_t nfree, double* d_out, cudaStream_t s);
void csr_mul(const DevCsr& a, const double* d_x, double* d_y, cudaStream_t s);
// Hex::new (hex.rs:218-297) for `n` box cells given by their 12 numbers each (the 3 sides, the
// 9 orthotropic constants): 576 values per cell into d_table.
void hex_elements(const double* d_keys, int64_t n, double* d_table, cudaStream_t s);
// The same with the 3 expansion coefficients after the constants (15 numbers per cell): the
// recovery record of each (HEX_MODES values, hex.cuh).
void hex_modes(const double* d_keys, int64_t n, double* d_modes, cudaStream_t s);
// The classes of `nel` box cells (8 corners each): the cells whose `width` numbers (the sides,
// the 9 constants of coef, with width 15 the 3 of expansion, which may be null: 0) are equal
// bit for bit share a class. `cls` gets each cell's class, `keys` the numbers of each class;
// returns the class count.
int64_t hex_classes(const double* d_xyz, const uint32_t* d_el, const double* d_coef,
                    const double* d_expansion, int width, int64_t nel, DevBuf<uint32_t>* cls,
                    DevBuf<double>* keys, cudaStream_t s);
// Throws the error of an assembly's device flag (0: none).
void assembly_flag(int b);

}  // namespace femgpu
