"""ctypes binding of libfemgpu.so (include/femgpu.h). Loading fails loudly when the library is
missing: there is no CPU path behind this package."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfemgpu.so")

# Status codes (femgpu.h).
OK, CANCELLED, NOT_CONVERGED, NOT_SPD, NEEDS_GRID, INVALID, CUDA, TOO_LARGE, PATTERN, MATERIAL, \
    TIMEOUT = range(11)

P1_HEAT, P1_ELASTIC, P2_ELASTIC, P2_MASS, P2_ELASTIC_ORTHO, HEX8_HEAT, HEX8_ELASTIC, HEX8_MASS = \
    range(8)
GATHER, COLOUR = 0, 1
FP64, MIXED = 0, 1


class FemError(RuntimeError):
    """A failure of the library: ``code`` is the femgpu.h status and ``str(e)`` the message (the
    reference's text where it has one, e.g. "cancelled")."""

    def __init__(self, code, message):
        super().__init__(message)
        self.code = code


class Unknowns_t(C.Structure):
    _fields_ = [
        ("kind", C.c_int),
        ("planes", C.c_void_p * 3),
        ("nplanes", C.c_size_t * 3),
        ("points", C.c_void_p),
        ("comp", C.c_void_p),
        ("xyz", C.c_void_p),
        ("p_cols", C.c_size_t),
        ("p_ptr", C.c_void_p),
        ("p_idx", C.c_void_p),
        ("p_val", C.c_void_p),
        ("coarse_xyz", C.c_void_p),
        ("coarse_comp", C.c_void_p),
    ]


class Crossover_t(C.Structure):
    _fields_ = [("rule", C.c_int), ("unknowns", C.c_size_t), ("flops", C.c_double),
                ("entries", C.c_uint64), ("flat", C.c_int)]


class Cells_t(C.Structure):
    _fields_ = [("count", C.c_size_t), ("origin", C.c_void_p), ("cls", C.c_void_p),
                ("matrices", C.c_void_p), ("nclass", C.c_size_t), ("mass", C.c_void_p)]


class Options_t(C.Structure):
    _fields_ = [("precision", C.c_int), ("degree", C.c_int), ("lower", C.c_double),
                ("sell_c", C.c_int), ("sell_sigma", C.c_int), ("coarsest", C.c_int),
                ("max_levels", C.c_int), ("graph", C.c_int), ("format", C.c_int),
                ("tail", C.c_int), ("launch", C.c_int), ("values", C.c_int),
                ("tiles", C.c_int), ("axes", C.c_int), ("stencil", C.c_int),
                ("smoother", C.c_int), ("cluster", C.c_int), ("l2", C.c_int),
                ("upper", C.c_double)]


class BatchStats_t(C.Structure):
    _fields_ = [("max_iterations", C.c_size_t), ("mean_iterations", C.c_double),
                ("max_residual", C.c_double), ("max_true_residual", C.c_double),
                ("seconds", C.c_double), ("launches", C.c_size_t),
                ("not_converged", C.c_size_t), ("restarts", C.c_size_t)]


class Stats_t(C.Structure):
    _fields_ = [("iterations", C.c_size_t), ("residual", C.c_double),
                ("true_residual", C.c_double), ("seconds", C.c_double),
                ("launches", C.c_size_t)]


class Energy_t(C.Structure):
    _fields_ = [("stored", C.c_double), ("fixed", C.c_double), ("gross", C.c_double)]


class ModesStats_t(C.Structure):
    _fields_ = [("iterations", C.c_size_t), ("solves", C.c_size_t),
                ("pcg_iterations", C.c_size_t), ("shift", C.c_double), ("seconds", C.c_double)]


class Peak_t(C.Structure):
    _fields_ = [("mises", C.c_double), ("element", C.c_int64), ("local", C.c_int32),
                ("point", C.c_uint32), ("singular", C.c_int32), ("pad", C.c_int32),
                ("regular_mises", C.c_double), ("regular_element", C.c_int64),
                ("regular_local", C.c_int32), ("regular_point", C.c_uint32)]


_lib = None

# Every symbol of include/femgpu.h with its signature.
class Outline_t(C.Structure):
    _fields_ = [("circle", C.c_int), ("ncorners", C.c_size_t), ("corners", C.c_void_p),
                ("centre", C.c_double * 2), ("radius", C.c_double)]


class Part_t(C.Structure):
    _fields_ = [("name", C.c_char_p), ("material", C.c_size_t), ("priority", C.c_int64),
                ("lo", C.c_double * 3), ("hi", C.c_double * 3), ("has_footprint", C.c_int),
                ("outline", Outline_t), ("nholes", C.c_size_t), ("holes", C.c_void_p)]


class Spacing_t(C.Structure):
    _fields_ = [("max_cell", C.c_double), ("max_growth", C.c_double), ("min_cells", C.c_size_t)]


class TetmeshCounts_t(C.Structure):
    _fields_ = [(k, C.c_size_t) for k in ("points", "tets", "faces", "face_circles", "circles",
                                           "triangles", "planes")]


class BoxgridCounts_t(C.Structure):
    _fields_ = [("planes", C.c_size_t * 3), ("grid_cells", C.c_size_t), ("points", C.c_size_t),
                ("cells", C.c_size_t), ("faces", C.c_size_t)]


class Convergence_t(C.Structure):
    _fields_ = [("iterations", C.c_size_t), ("residual", C.c_double)]


PRECONDITION_FN = C.CFUNCTYPE(None, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_size_t,
                              C.c_void_p)
PRECONDITION_DEVICE_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p,
                                     C.c_void_p)

CLASSIFY_FN = C.CFUNCTYPE(C.c_uint32, C.POINTER(C.c_double), C.c_void_p)

SIGNATURES = {
    "femgpu_prism_mesh": (C.c_int, [C.c_void_p, C.c_size_t, C.c_int, C.POINTER(Spacing_t),
                                    C.c_size_t, C.c_char_p, C.c_int, C.c_void_p, C.c_size_t,
                                    C.POINTER(C.c_void_p)]),
    "femgpu_tetmesh_sizes": (C.c_int, [C.c_void_p, C.POINTER(TetmeshCounts_t)]),
    "femgpu_tetmesh_copy": (C.c_int, [C.c_void_p] + [C.c_void_p] * 9),
    "femgpu_tetmesh_device": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p),
                                        C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]),
    "femgpu_tetmesh_free": (None, [C.c_void_p]),
    "femgpu_axis_planes": (C.c_int, [C.c_void_p, C.c_size_t, C.c_int, C.POINTER(Spacing_t),
                                     C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t,
                                     C.POINTER(C.c_size_t)]),
    "femgpu_mesh2d": (C.c_int, [C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.c_double,
                                C.c_double, C.c_int, CLASSIFY_FN, C.c_void_p,
                                C.POINTER(C.c_void_p)]),
    "femgpu_mesh2_sizes": (C.c_int, [C.c_void_p, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t),
                                     C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
    "femgpu_mesh2_copy": (C.c_int, [C.c_void_p] + [C.c_void_p] * 7),
    "femgpu_mesh2_free": (None, [C.c_void_p]),
    "femgpu_split_prism": (C.c_int, [C.c_void_p, C.c_void_p]),
    "femgpu_csr_diagonal": (C.c_int, [C.c_void_p, C.c_void_p]),
    "femgpu_rect_upload": (C.c_int, [C.c_size_t, C.c_size_t, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.POINTER(C.c_void_p)]),
    "femgpu_rect_mul": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "femgpu_rect_mul_transpose": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "femgpu_rect_galerkin": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_void_p)]),
    "femgpu_rect_free": (None, [C.c_void_p]),
    "femgpu_pcg": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, PRECONDITION_FN, C.c_void_p,
                             C.c_double, C.c_size_t, C.c_void_p, C.POINTER(Convergence_t)]),
    "femgpu_pcg_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, PRECONDITION_DEVICE_FN,
                                    C.c_void_p, C.c_double, C.c_size_t, C.c_void_p, C.c_void_p,
                                    C.POINTER(Convergence_t)]),
    "femgpu_box_grid": (C.c_int, [C.c_void_p, C.c_size_t, C.POINTER(Spacing_t), C.c_void_p,
                                  C.c_void_p, C.c_size_t, C.c_char_p, C.POINTER(C.c_void_p)]),
    "femgpu_boxgrid_sizes": (C.c_int, [C.c_void_p, C.POINTER(BoxgridCounts_t)]),
    "femgpu_boxgrid_copy": (C.c_int, [C.c_void_p] + [C.c_void_p] * 9),
    "femgpu_boxgrid_device": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p),
                                        C.POINTER(C.c_void_p)]),
    "femgpu_boxgrid_free": (None, [C.c_void_p]),
    "femgpu_last_error": (C.c_size_t, [C.c_char_p, C.c_size_t]),
    "femgpu_version": (C.c_char_p, []),
    "femgpu_assemble": (C.c_int, [C.c_int, C.c_int, C.c_size_t, C.c_void_p, C.c_size_t,
                                  C.c_void_p, C.c_void_p, C.POINTER(C.c_void_p)]),
    "femgpu_assemble_device": (C.c_int, [C.c_int, C.c_int, C.c_size_t, C.c_void_p, C.c_size_t,
                                         C.c_void_p, C.c_void_p, C.POINTER(C.c_void_p)]),
    "femgpu_pattern": (C.c_int, [C.c_size_t, C.c_size_t, C.c_int, C.c_void_p,
                                 C.POINTER(C.c_void_p)]),
    "femgpu_colour": (C.c_int, [C.c_size_t, C.c_size_t, C.c_int, C.c_void_p, C.c_void_p,
                                C.POINTER(C.c_int)]),
    "femgpu_quadratic": (C.c_int, [C.c_size_t, C.c_size_t, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.POINTER(C.c_size_t)]),
    "femgpu_csr_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
    "femgpu_csr_download": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "femgpu_csr_upload": (C.c_int, [C.c_size_t, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.POINTER(C.c_void_p)]),
    "femgpu_csr_submatrix": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t,
                                       C.POINTER(C.c_void_p)]),
    "femgpu_csr_mul": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "femgpu_reduced_rhs": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_size_t, C.c_void_p]),
    "femgpu_csr_free": (None, [C.c_void_p]),
    "femgpu_reduced_rhs_noalloc": (C.c_int, [C.c_size_t, C.c_void_p, C.c_void_p, C.c_void_p,
                                             C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t,
                                             C.c_void_p, C.c_void_p]),
    "femgpu_prolongation": (C.c_int, [C.c_size_t, C.c_void_p, C.c_size_t, C.c_size_t,
                                      C.c_void_p, C.c_size_t, C.c_void_p,
                                      C.POINTER(C.c_size_t), C.POINTER(C.c_size_t), C.c_void_p,
                                      C.c_void_p, C.c_void_p, C.c_void_p]),
    "femgpu_solver_new": (C.c_int, [C.c_void_p, C.POINTER(Unknowns_t), C.c_int,
                                    C.POINTER(Crossover_t), C.POINTER(Options_t),
                                    C.POINTER(C.c_void_p)]),
    "femgpu_solver_new_cells": (C.c_int, [C.c_void_p, C.POINTER(Unknowns_t), C.c_int,
                                          C.POINTER(Crossover_t), C.POINTER(Options_t),
                                          C.POINTER(Cells_t), C.POINTER(C.c_void_p)]),
    "femgpu_hex_elements": (C.c_int, [C.c_size_t, C.c_void_p, C.c_void_p]),
    "femgpu_symbolic_counts": (C.c_int, [C.c_void_p, C.POINTER(Unknowns_t),
                                         C.POINTER(C.c_uint64), C.POINTER(C.c_double)]),
    "femgpu_hex_mass": (C.c_int, [C.c_size_t, C.c_void_p, C.c_void_p, C.c_void_p]),
    "femgpu_coarse_matrix": (C.c_int, [C.c_void_p, C.POINTER(Unknowns_t), C.POINTER(Cells_t),
                                       C.c_int, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t),
                                       C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_void_p]),
    "femgpu_solver_set_max_iter": (C.c_int, [C.c_void_p, C.c_size_t]),
    "femgpu_solver_set_wait_limit": (C.c_int, [C.c_void_p, C.c_uint32]),
    "femgpu_solver_set_tol": (C.c_int, [C.c_void_p, C.c_double]),
    "femgpu_solver_method": (C.c_int, [C.c_void_p]),
    "femgpu_solver_levels": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    "femgpu_solver_bytes": (C.c_size_t, [C.c_void_p]),
    "femgpu_solver_describe": (C.c_size_t, [C.c_void_p, C.c_char_p, C.c_size_t]),
    "femgpu_solver_breakdown": (C.c_size_t, [C.c_void_p, C.c_char_p, C.c_size_t]),
    "femgpu_solver_solve": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.POINTER(Stats_t)]),
    "femgpu_solver_solve_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                             C.POINTER(Stats_t)]),
    "femgpu_solver_solve_zero": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                             C.POINTER(Stats_t)]),
    "femgpu_solver_precondition_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "femgpu_solver_free": (None, [C.c_void_p]),
    "femgpu_solver_stream": (C.c_void_p, [C.c_void_p]),
    "femgpu_solver_kernel_time": (C.c_int, [C.c_void_p, C.c_int, C.c_int,
                                            C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "femgpu_server_new": (C.c_int, [C.c_int, C.c_size_t, C.POINTER(C.c_void_p)]),
    "femgpu_server_reserve": (C.c_int, [C.c_void_p, C.c_size_t]),
    "femgpu_server_put": (C.c_int, [C.c_void_p, C.c_uint64, C.c_void_p]),
    "femgpu_server_has": (C.c_int, [C.c_void_p, C.c_uint64]),
    "femgpu_server_submit": (C.c_int, [C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p,
                                       C.POINTER(C.c_uint64)]),
    "femgpu_server_wait": (C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(Stats_t),
                                     C.POINTER(C.c_double)]),
    "femgpu_server_resident_bytes": (C.c_size_t, [C.c_void_p]),
    "femgpu_server_resident_count": (C.c_size_t, [C.c_void_p]),
    "femgpu_server_free": (None, [C.c_void_p]),
    "femgpu_batch_new": (C.c_int, [C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                   C.POINTER(C.c_void_p)]),
    "femgpu_batch_set_tol": (C.c_int, [C.c_void_p, C.c_double]),
    "femgpu_batch_set_max_iter": (C.c_int, [C.c_void_p, C.c_size_t]),
    "femgpu_batch_systems": (C.c_int, [C.c_void_p, C.c_void_p]),
    "femgpu_batch_levels": (C.c_int, [C.c_void_p, C.c_void_p]),
    "femgpu_batch_describe": (C.c_int, [C.c_void_p, C.c_char_p, C.c_size_t]),
    "femgpu_batch_solve": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.POINTER(BatchStats_t)]),
    "femgpu_batch_solve_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                            C.POINTER(BatchStats_t)]),
    "femgpu_batch_segments": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_void_p]),
    "femgpu_batch_kernel_time": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_double),
                                           C.POINTER(C.c_double)]),
    "femgpu_batch_bytes": (C.c_size_t, [C.c_void_p]),
    "femgpu_batch_stream": (C.c_void_p, [C.c_void_p]),
    "femgpu_batch_free": (None, [C.c_void_p]),
    "femgpu_stream_new": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "femgpu_stream_submit": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.POINTER(C.c_uint64)]),
    "femgpu_stream_wait": (C.c_int, [C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p]),
    "femgpu_stream_counts": (C.c_int, [C.c_void_p, C.POINTER(C.c_size_t),
                                       C.POINTER(C.c_size_t)]),
    "femgpu_stream_free": (None, [C.c_void_p]),
    "femgpu_modes": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.c_double,
                               C.POINTER(Unknowns_t), C.c_int, C.POINTER(Crossover_t),
                               C.POINTER(Options_t), C.c_void_p, C.c_void_p, C.c_void_p,
                               C.POINTER(ModesStats_t)]),
    "femgpu_modes_cells": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.c_double,
                               C.POINTER(Unknowns_t), C.c_int, C.POINTER(Crossover_t),
                               C.POINTER(Options_t), C.POINTER(Cells_t), C.c_void_p, C.c_void_p, C.c_void_p,
                               C.POINTER(ModesStats_t)]),
    "femgpu_dense_generalized": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p,
                                           C.c_void_p]),
    "femgpu_transient_new": (C.c_int, [C.c_void_p, C.c_void_p, C.c_double, C.c_void_p,
                                       C.c_size_t, C.POINTER(Unknowns_t), C.c_int,
                                       C.POINTER(Crossover_t), C.POINTER(Options_t),
                                       C.POINTER(C.c_void_p)]),
    "femgpu_transient_solver": (C.c_void_p, [C.c_void_p]),
    "femgpu_transient_run": (C.c_int, [C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p,
                                       C.c_size_t, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.POINTER(Stats_t)]),
    "femgpu_transient_free": (None, [C.c_void_p]),
    "femgpu_recovery_new": (C.c_int, [C.c_size_t, C.c_void_p, C.c_size_t, C.c_void_p,
                                      C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t,
                                      C.c_void_p, C.POINTER(C.c_void_p)]),
    "femgpu_recovery_new_hex": (C.c_int, [C.c_size_t, C.c_void_p, C.c_size_t, C.c_void_p,
                                      C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t,
                                      C.c_void_p, C.POINTER(C.c_void_p)]),
    "femgpu_hex_loads": (C.c_int, [C.c_size_t, C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "femgpu_reactions": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_size_t, C.c_void_p, C.c_double, C.c_void_p,
                                   C.c_void_p, C.c_void_p, C.c_void_p]),
    "femgpu_recovery_probes": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_size_t, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "femgpu_recovery_run": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "femgpu_recovery_run_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                             C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "femgpu_recovery_last_time": (C.c_int, [C.c_void_p, C.POINTER(C.c_double),
                                            C.POINTER(C.c_double)]),
    "femgpu_recovery_bytes": (C.c_size_t, [C.c_void_p]),
    "femgpu_recovery_stream": (C.c_void_p, [C.c_void_p]),
    "femgpu_recovery_free": (None, [C.c_void_p]),
}


def lib():
    """The loaded library; raises when libfemgpu.so is missing (build it with
    ``python -m femahoy_b200.build``)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with python -m femahoy_b200.build")
        handle = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(handle, name)
            f.restype = res
            f.argtypes = args
        _lib = handle
    return _lib


def check(status):
    if status != OK:
        buf = C.create_string_buffer(1024)
        lib().femgpu_last_error(buf, 1024)
        raise FemError(status, buf.value.decode())


def ptr(a):
    """The data pointer of a contiguous numpy array (None for None)."""
    if a is None:
        return None
    return a.ctypes.data_as(C.c_void_p)


def arr(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)
