"""ctypes binding of libcurvenet_b200.so (the C ABI in include/curvenet_b200.h).

The library is built in-tree (tool_godot_curvenet_b200/lib/).  There is no
fallback: importing the binding without the built library raises.
"""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libcurvenet_b200.so")

CN_OK, CN_MAX_ITER, CN_SINGULAR_COMPONENT, CN_NONPOS_PIVOT, CN_NAN = 0, 1, 2, 3, 4
CN_BREAKDOWN, CN_TIMEOUT, CN_BAD_INPUT, CN_CUDA_ERROR, CN_NO_DEVICE = 5, 6, 7, 8, 9
PRECOND_JACOBI, PRECOND_IC0, PRECOND_HSC, PRECOND_BSSOR = 0, 1, 2, 3
ORDER_NATURAL, ORDER_COLOR, ORDER_AUTO = 0, 1, 2
LAPLACIAN_COT, LAPLACIAN_ROBUST = 0, 1
PREC_FP64, PREC_MIXED = 0, 1
MODE_HARMONIC, MODE_DEFORM, MODE_RHS = 0, 1, 2
ALGO_FUSED, ALGO_PLAIN, ALGO_CLASSIC, ALGO_PIPELINED, ALGO_SINGLE = 0, 1, 2, 3, 4


class MeshDesc(C.Structure):
    _fields_ = [("n_verts", C.c_int32), ("n_tris", C.c_int32),
                ("positions", C.POINTER(C.c_double)), ("tris", C.POINTER(C.c_int32)),
                ("n_handles", C.c_int32), ("handles", C.POINTER(C.c_int32))]


class BuildOpts(C.Structure):
    _fields_ = [("precond", C.c_int32), ("ordering", C.c_int32), ("laplacian", C.c_int32),
                ("mollify_delta", C.c_double), ("device", C.c_int32), ("max_rhs", C.c_int32),
                ("tune", C.c_int32), ("lanes", C.c_int32), ("block", C.c_int32),
                ("grid", C.c_int32), ("hsc_tail_rows", C.c_int32), ("hsc_theta", C.c_double)]


class SolveOpts(C.Structure):
    _fields_ = [("precision", C.c_int32), ("mode", C.c_int32), ("algo", C.c_int32),
                ("tol", C.c_double), ("max_iter", C.c_int32), ("max_refine", C.c_int32),
                ("inner_tol", C.c_double), ("warm_start", C.c_int32), ("wait_limit_ms", C.c_double)]


class CurvenetDesc(C.Structure):
    _fields_ = [("n_curves", C.c_int32), ("n_segments", C.c_int32), ("n_samples", C.c_int32),
                ("rest_cp", C.POINTER(C.c_double)), ("sample_tau", C.POINTER(C.c_double)),
                ("closed", C.POINTER(C.c_int32)), ("n_nodes", C.c_int32), ("node_ptr", C.POINTER(C.c_int32)),
                ("node_ends", C.POINTER(C.c_int32)), ("handle_curve", C.POINTER(C.c_int32)),
                ("handle_sample", C.POINTER(C.c_int32)), ("handle_side", C.POINTER(C.c_int32))]


class BatchStats(C.Structure):
    _fields_ = [("status", C.c_int32), ("n_meshes", C.c_int32), ("n_failed", C.c_int32),
                ("max_iterations", C.c_int32), ("total_iterations", C.c_int64),
                ("max_rel_residual", C.c_double), ("device_ms", C.c_double)]


class SolveStats(C.Structure):
    _fields_ = [("status", C.c_int32), ("iterations", C.c_int32), ("refinements", C.c_int32),
                ("k", C.c_int32), ("rel_residual", C.c_double * 32),
                ("max_rel_residual", C.c_double), ("device_ms", C.c_double)]


_P = C.c_void_p
_I32P = C.POINTER(C.c_int32)
_DP = C.POINTER(C.c_double)

# name -> (restype, argtypes); every symbol the header declares
SIGNATURES = {
    "cn_default_build_opts": (None, [C.POINTER(BuildOpts)]),
    "cn_default_solve_opts": (None, [C.POINTER(SolveOpts)]),
    "cn_status_string": (C.c_char_p, [C.c_int32]),
    "cn_last_error": (C.c_char_p, []),
    "cn_cut_mesh": (C.c_int, [C.c_int32, C.c_int32, _I32P, C.c_int32, _I32P, _I32P, _I32P, _I32P, _I32P]),
    "cn_build": (C.c_int, [C.POINTER(MeshDesc), C.POINTER(BuildOpts), C.POINTER(_P)]),
    "cn_halfedges": (C.c_int, [C.c_int32, C.c_int32, _I32P, _I32P, _I32P]),
    "cn_cut_mesh_gpu": (C.c_int, [C.c_int32, C.c_int32, _I32P, C.c_int32, _I32P, _I32P, _I32P, _I32P, _I32P]),
    "cn_subdivide_edges": (C.c_int, [_I32P, _I32P, C.c_int32, _I32P]),
    "cn_split_faces": (C.c_int, [_I32P, _I32P, C.c_int32, _I32P, _I32P]),
    "cn_insert_cracks": (C.c_int, [_I32P, _I32P, C.c_int32, _I32P]),
    "cn_destroy": (None, [_P]),
    "cn_solve": (C.c_int, [_P, C.c_int32, _DP, _DP, _DP, C.POINTER(SolveOpts), C.POINTER(SolveStats)]),
    "cn_solve_device": (C.c_int, [_P, C.c_int32, _P, _P, C.POINTER(SolveOpts), C.POINTER(SolveStats)]),
    "cn_stream": (_P, [_P]),
    "cn_system_info": (C.c_int, [_P, C.POINTER(C.c_int64)]),
    "cn_export_csr": (C.c_int, [_P, _I32P, _I32P, _I32P, _DP]),
    "cn_export_factor": (C.c_int, [_P, _I32P, _I32P, _DP]),
    "cn_export_k": (C.c_int, [_P, _I32P, _I32P, _DP]),
    "cn_solve_deformation": (C.c_int, [_P, _DP, _DP, _DP, C.POINTER(SolveOpts), C.POINTER(SolveStats)]),
    "cn_ddm_bind": (C.c_int, [_P, C.c_int32, C.c_double, C.c_int32, C.POINTER(SolveOpts), _I32P, _DP]),
    "cn_lbs_matvec_device": (C.c_int, [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_void_p, C.c_void_p, C.c_void_p]),
    "cn_spmv_device": (C.c_int, [_P, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p]),
    "cn_set_launch": (C.c_int, [_P, C.c_int32, C.c_int32, C.c_int32]),
    "cn_autotune": (C.c_int, [_P, C.c_int32, _P, C.POINTER(SolveOpts), C.c_int32, _DP, _I32P]),
    "cn_hsc_info": (C.c_int, [_P, _I32P, _I32P, _I32P, _I32P, _I32P]),
    "cn_bind_curves": (C.c_int, [_P, C.c_int32, C.c_int32, _DP, _I32P, _DP]),
    "cn_deform": (C.c_int, [_P, _DP, _DP, _DP, C.POINTER(SolveOpts), C.POINTER(SolveStats)]),
    "cn_adjoint": (C.c_int, [_P, _DP, _DP, _DP, C.POINTER(SolveOpts), C.POINTER(SolveStats)]),
    "cn_bind_curvenet": (C.c_int, [_P, C.POINTER(CurvenetDesc)]),
    "cn_curvenet_constraints_device": (C.c_int, [_P, C.c_int32, _P, _P, _P]),
    "cn_curvenet_constraints": (C.c_int, [_P, C.c_int32, _DP, _DP, _DP]),
    "cn_deform_curvenet": (C.c_int, [_P, _DP, _DP, C.POINTER(SolveOpts), C.POINTER(SolveStats)]),
    "cn_build_batch": (C.c_int, [C.POINTER(MeshDesc), C.c_int32, C.POINTER(BuildOpts), C.c_int32, C.c_int32,
                                 C.c_int32, C.POINTER(_P)]),
    "cn_destroy_batch": (None, [_P]),
    "cn_solve_batch": (C.c_int, [_P, _DP, _DP, C.POINTER(SolveOpts), C.POINTER(BatchStats)]),
    "cn_solve_batch_device": (C.c_int, [_P, _P, _P, C.POINTER(SolveOpts), C.POINTER(BatchStats)]),
    "cn_batch_stream": (_P, [_P]),
    "cn_batch_info": (C.c_int, [_P, C.POINTER(C.c_int64)]),
    "cn_batch_offsets": (C.c_int, [_P, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "cn_batch_mesh_stats": (C.c_int, [_P, _I32P, _I32P, _DP, _I32P]),
    "cn_batch_set_lanes": (C.c_int, [_P, C.c_int32, _I32P, _I32P]),
    "cn_batch_lanes": (C.c_int, [_P, _I32P]),
    "cn_pcg_csr_noalloc": (C.c_int, [C.c_int32, _P, _P, _P, C.c_int32, _P, _P, C.c_double, C.c_int32, _P,
                                     C.POINTER(SolveStats)]),
    "cn_pcg_csr_noalloc_last_stats": (C.c_int, [C.POINTER(SolveStats)]),
}

_lib = None


def lib():
    """Load the library once; raise if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'` "
                "(there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def last_error():
    return lib().cn_last_error().decode()


def status_string(s):
    return lib().cn_status_string(int(s)).decode()
