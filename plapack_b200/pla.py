"""ctypes binding of libplapack_b200.so (the C ABI declared in include/PLA.h).

The functions keep the reference's names and argument order (PLA_Init,
PLA_Temp_create, PLA_Matrix_create, PLA_API_axpy_matrix_to_global, PLA_LU, ...);
objects are opaque handles whose data lives in device memory.  A few helpers
at the bottom move numpy arrays in and out through the reference's own fill
and extract calls.

Importing this module requires the built library; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libplapack_b200.so")

# ---- constants (include/PLA.h, same values as the reference's PLA_define.h)
MPI_COMM_NULL, MPI_COMM_WORLD = 0, 1
MPI_CHAR, MPI_INT, MPI_FLOAT, MPI_DOUBLE = 1, 3, 4, 5
PLA_VECTOR, PLA_MVECTOR, PLA_MATRIX, PLA_MSCALAR, PLA_PVECTOR, PLA_PMVECTOR = 11, 12, 13, 14, 15, 16
PLA_NO_TRANSPOSE, PLA_TRANSPOSE, PLA_CONJUGATE_TRANSPOSE = 21, 22, 23
PLA_NO_TRANS, PLA_TRANS = 21, 22
PLA_ALL_ROWS, PLA_ALL_COLS = -31, -32
PLA_SIDE_TOP, PLA_SIDE_BOTTOM, PLA_SIDE_LEFT, PLA_SIDE_RIGHT = 41, 42, 43, 44
PLA_UPPER_TRIANGULAR, PLA_LOWER_TRIANGULAR = 51, 52
PLA_OP_PAN_PAN, PLA_OP_ALL_ALG = 83, 87
PLA_VERSION_A, PLA_VERSION_B, PLA_VERSION_C = 100, 200, 300
PLA_PROJ_ONTO_COL, PLA_PROJ_ONTO_ROW = 91, 92
PLA_UNIT_DIAG, PLA_NONUNIT_DIAG = 101, 102
PLA_SUCCESS, PLA_ALIGN_FIRST, PLA_DIM_ALL = 0, -200, -201
PLA_ERROR = -1000

PLA_B200_PREC_BF16, PLA_B200_PREC_FP16, PLA_B200_PREC_FP32, PLA_B200_PREC_FP64 = 1, 2, 3, 4
PLA_B200_PREC_FP8 = 5
PLA_B200_PREC_BF16X6 = 6
PLA_B200_PREC_BF16X3 = 7
PLA_B200_IR_LU, PLA_B200_IR_GMRES = 1, 2
PLA_B200_PIVOT_PARTIAL, PLA_B200_PIVOT_TOURNAMENT = 0, 1

_DT = {np.dtype(np.float64): MPI_DOUBLE, np.dtype(np.float32): MPI_FLOAT,
       np.dtype(np.int32): MPI_INT}
_NP = {v: k for k, v in _DT.items()}

Obj = ctypes.c_void_p
Templ = ctypes.c_void_p
_i, _vp, _d = ctypes.c_int, ctypes.c_void_p, ctypes.c_double
_pi, _pobj = ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_void_p)


class PhaseTimes(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in
                ("total_ms", "panel_ms", "swap_ms", "trsm_ms", "update_ms", "solve_ms", "refine_ms",
                 "convert_ms")] + [("update_launches", ctypes.c_int),
                                   ("interchanges", ctypes.c_longlong)]


class MixedParams(ctypes.Structure):
    _fields_ = [("precision", _i), ("refinement", _i), ("max_iterations", _i),
                ("gmres_restart", _i), ("nb", _i), ("escalate", _i), ("tol", _d),
                ("panel_pivoting", _i)]


class MixedReport(ctypes.Structure):
    _fields_ = [("converged", _i), ("iterations", _i), ("inner_iterations", _i), ("info", _i),
                ("backward_error", _d), ("factor_ms", _d), ("refine_ms", _d),
                ("precision_used", _i), ("factorizations", _i)]


class BatchInstance(ctypes.Structure):
    _fields_ = [("n", _i), ("nrhs", _i), ("kind", _i), ("A", _vp), ("B", _vp),
                ("pivots", ctypes.POINTER(ctypes.c_int))]


# name -> argtypes (restype int unless listed in _RESTYPE)
_SIGS = {
    "PLA_Init": [_i], "PLA_Finalize": [], "PLA_Initialized": [_pi],
    "PLA_Comm_1D_to_2D": [_i, _i, _i, _pi],
    "PLA_Temp_create": [_i, _i, _pobj], "PLA_Temp_free": [_pobj],
    "PLA_Temp_nb": [Templ, _pi],
    "pla_Environ_set_nb_alg": [_i, _i], "PLA_Environ_nb_alg": [_i, Templ, _pi],
    "PLA_Set_error_checking": [_i, _i, _i, _i], "PLA_Get_error_checking": [_pi, _pi, _pi, _pi],
    "PLA_Matrix_create": [_i, _i, _i, Templ, _i, _i, _pobj],
    "PLA_Mvector_create": [_i, _i, _i, Templ, _i, _pobj],
    "PLA_Mscalar_create": [_i, _i, _i, _i, _i, Templ, _pobj],
    "PLA_Pmvector_create": [_i, _i, _i, _i, _i, Templ, _i, _pobj],
    "PLA_Matrix_create_conf_to": [Obj, _pobj],
    "PLA_Mvector_create_conf_to": [Obj, _i, _pobj],
    "PLA_Mscalar_create_conf_to": [Obj, _i, _i, _pobj],
    "PLA_Create_constants_conf_to": [Obj, _pobj, _pobj, _pobj],
    "PLA_Obj_free": [_pobj],
    "PLA_Obj_view": [Obj, _i, _i, _i, _i, _pobj], "PLA_Obj_view_all": [Obj, _pobj],
    "PLA_Obj_split_4": [Obj, _i, _i, _pobj, _pobj, _pobj, _pobj],
    "PLA_Obj_horz_split_2": [Obj, _i, _pobj, _pobj], "PLA_Obj_vert_split_2": [Obj, _i, _pobj, _pobj],
    "PLA_Obj_view_shift": [Obj, _i, _i, _i, _i],
    "PLA_Obj_objtype": [Obj, _pi], "PLA_Obj_datatype": [Obj, _pi],
    "PLA_Obj_global_length": [Obj, _pi], "PLA_Obj_global_width": [Obj, _pi],
    "PLA_Obj_local_length": [Obj, _pi], "PLA_Obj_local_width": [Obj, _pi],
    "PLA_Obj_local_ldim": [Obj, _pi], "PLA_Obj_local_buffer": [Obj, _pobj],
    "PLA_Obj_set_to_zero": [Obj], "PLA_Obj_set_to_one": [Obj], "PLA_Obj_set_to_minus_one": [Obj],
    "PLA_Obj_set": [Obj, _i, _vp],
    "PLA_Obj_get_local_contents": [Obj, _i, _pi, _pi, _vp, _i, _i],
    "PLA_Obj_set_local_contents": [_i, _i, _i, _vp, _i, _i, Obj],
    "PLA_Copy": [Obj, Obj],
    "PLA_API_begin": [], "PLA_API_end": [], "PLA_Obj_API_open": [Obj], "PLA_Obj_API_close": [Obj],
    "PLA_API_axpy_matrix_to_global": [_i, _i, _vp, _vp, _i, Obj, _i, _i],
    "PLA_API_axpy_global_to_matrix": [_i, _i, _vp, Obj, _i, _i, _vp, _i],
    "PLA_API_axpy_vector_to_global": [_i, _vp, _vp, _i, Obj, _i],
    "PLA_API_axpy_global_to_vector": [_i, _vp, Obj, _i, _vp, _i],
    "PLA_LU": [Obj, Obj], "PLA_LU_info": [Obj, Obj, _pi],
    "PLA_LU_linpack": [Obj, Obj], "PLA_LU_linpack_right": [_i, Obj, Obj],
    "PLA_LU_right": [_i, Obj, Obj], "PLA_LU_right_mv": [Obj, Obj, Obj],
    "PLA_Gemm_x": [_i, _i, _i, Obj, Obj, Obj, Obj, Obj],
    "PLA_Timings_initialize": [], "PLA_Timings_print": [], "PLA_Timings_average": [],
    "PLA_Axpy": [Obj, Obj, Obj], "PLA_Nrm2": [Obj, Obj], "PLA_Shift": [Obj, _i, _vp],
    "PLA_Local_axpy": [Obj, Obj, Obj], "PLA_Local_nrm2": [Obj, Obj],
    "PLA_malloc": [ctypes.c_size_t], "PLA_calloc": [ctypes.c_size_t, ctypes.c_size_t],
    "PLA_free": [_vp], "PLA_Total_size_malloced": [], "PLA_Max_size_malloced": [],
    "PLA_OOC_Matrix_create_without_fd": [_i, _i, _i, Templ, _i, _i, _pobj],
    "PLA_Obj_attach_fd": [Obj, _i, _i, _i], "PLA_File_create": [ctypes.c_char_p, _i, _i, _pi],
    "PLA_File_open": [ctypes.c_char_p, _i, _i, _pi], "PLA_File_close": [_i],
    "PLA_File_unlink": [ctypes.c_char_p], "PLA_File_stats_start": [], "PLA_File_stats_stop": [],
    "PLA_OOC_Chol": [_i, _i, Obj],
    "PLA_B200_file_stats": [ctypes.POINTER(ctypes.c_double)] * 4,
    "PLA_Apply_pivots_to_rows": [Obj, Obj], "PLA_General_solve": [Obj, Obj, Obj],
    "PLA_Chol": [_i, Obj], "PLA_Pos_def_solve": [Obj, Obj],
    "PLA_Trsv": [_i, _i, _i, Obj, Obj], "PLA_Trsm": [_i, _i, _i, _i, Obj, Obj, Obj],
    "PLA_Gemm": [_i, _i, Obj, Obj, Obj, Obj, Obj], "PLA_Gemv": [_i, Obj, Obj, Obj, Obj, Obj],
    "PLA_Iamax": [Obj, Obj, Obj],
    "PLA_Syrk_perform_local_part": [_i, Obj, Obj, Obj, Obj, Obj],
    "PLA_Local_gemm": [_i, _i, Obj, Obj, Obj, Obj, Obj],
    "PLA_Local_trsm": [_i, _i, _i, _i, Obj, Obj, Obj],
    "PLA_Local_syrk": [_i, _i, Obj, Obj, Obj, Obj],
    "PLA_Local_iamax": [Obj, _pi, _vp], "PLA_Local_scal": [Obj, Obj],
    "PLA_Local_inv_scal": [Obj, Obj], "PLA_Local_swap": [Obj, Obj], "PLA_Local_copy": [Obj, Obj],
    "PLA_Local_ger": [Obj, Obj, Obj, Obj], "PLA_Local_gemv": [_i, Obj, Obj, Obj, Obj, Obj],
    "PLA_Local_trsv": [_i, _i, _i, Obj, Obj], "PLA_Local_chol": [_i, Obj],
    "PLA_Last_error": [ctypes.c_char_p, _i], "PLA_Clear_error": [],
    "PLA_B200_set_stream": [_vp], "PLA_B200_get_stream": [],
    "PLA_B200_phase_times": [ctypes.POINTER(PhaseTimes)], "PLA_B200_set_phase_timing": [_i],
    "PLA_B200_reset_phase_times": [], "PLA_B200_kernel_launches": [],
    "PLA_Mixed_params_default": [ctypes.POINTER(MixedParams)],
    "PLA_General_solve_mixed": [Obj, Obj, ctypes.POINTER(MixedParams), ctypes.POINTER(MixedReport)],
    "PLA_Pos_def_solve_mixed": [Obj, Obj, ctypes.POINTER(MixedParams), ctypes.POINTER(MixedReport)],
    "PLA_General_solve_mixed_host": [Obj, _vp, _i, Obj, ctypes.POINTER(MixedParams),
                                     ctypes.POINTER(MixedReport)],
    "PLA_Batch_plan_create": [_i, _i, ctypes.POINTER(BatchInstance), _vp, _i, _pobj],
    "PLA_Batch_plan_execute": [_vp], "PLA_Batch_plan_free": [_pobj],
    "PLA_Batched_factor_solve": [_i, _i, ctypes.POINTER(BatchInstance), _vp],
    "PLA_Batched_factor_solve_loop": [_i, _i, ctypes.POINTER(BatchInstance)],
    "PLA_Obj_set_local_contents_device": [_vp, _i, Obj],
    "PLA_Obj_get_local_contents_device": [Obj, _vp, _i],
}
_RESTYPE = {"PLA_B200_get_stream": _vp, "PLA_Mixed_params_default": None,
            "PLA_B200_kernel_launches": ctypes.c_long, "PLA_malloc": _vp, "PLA_calloc": _vp,
            "PLA_free": _vp}


class PLAError(RuntimeError):
    pass


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    if not os.path.exists(path):
        raise PLAError(f"{path} is missing: build it with `make -C plapack_b200/csrc`")
    lib = ctypes.CDLL(path)
    for name, args in _SIGS.items():
        try:
            fn = getattr(lib, name)
        except AttributeError:
            continue  # reported by the export test, not at import
        fn.argtypes = args
        fn.restype = _RESTYPE.get(name, _i)
    return lib


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        _lib = load()
    return _lib


def last_error() -> str:
    buf = ctypes.create_string_buffer(512)
    lib().PLA_Last_error(buf, 512)
    return buf.value.decode()


def check(rc: int, what: str = "") -> int:
    if rc == PLA_ERROR:
        raise PLAError(f"{what}: {last_error()}")
    return rc


class Session:
    """PLA_Init + PLA_Temp_create on a 1x1 mesh, as TEST/test_lu.c:68-77 does."""

    def __init__(self, nb_distr: int = 128, nb_alg: int = 128, error_checking: int = 1):
        self.lib = lib()
        init = ctypes.c_int(0)
        self.lib.PLA_Initialized(ctypes.byref(init))
        if not init.value:
            comm = ctypes.c_int(0)
            check(self.lib.PLA_Comm_1D_to_2D(MPI_COMM_WORLD, 1, 1, ctypes.byref(comm)), "comm")
            check(self.lib.PLA_Init(comm.value), "PLA_Init")
        self.lib.pla_Environ_set_nb_alg(PLA_OP_ALL_ALG, nb_alg)
        self.lib.PLA_Set_error_checking(error_checking, error_checking, 0, 0)
        self.templ = ctypes.c_void_p()
        check(self.lib.PLA_Temp_create(nb_distr, 0, ctypes.byref(self.templ)), "PLA_Temp_create")

    def set_nb_alg(self, nb: int) -> None:
        check(self.lib.pla_Environ_set_nb_alg(PLA_OP_ALL_ALG, nb), "nb_alg")

    # --- object helpers -----------------------------------------------------
    def matrix(self, m: int, n: int, dtype=np.float64) -> ctypes.c_void_p:
        h = ctypes.c_void_p()
        check(self.lib.PLA_Matrix_create(_DT[np.dtype(dtype)], m, n, self.templ, PLA_ALIGN_FIRST,
                                         PLA_ALIGN_FIRST, ctypes.byref(h)), "Matrix_create")
        return h

    def mvector(self, m: int, n: int = 1, dtype=np.float64) -> ctypes.c_void_p:
        h = ctypes.c_void_p()
        check(self.lib.PLA_Mvector_create(_DT[np.dtype(dtype)], m, n, self.templ, PLA_ALIGN_FIRST,
                                          ctypes.byref(h)), "Mvector_create")
        return h

    def scalar(self, value: float, dtype=np.float64) -> ctypes.c_void_p:
        h = ctypes.c_void_p()
        check(self.lib.PLA_Mscalar_create(_DT[np.dtype(dtype)], PLA_ALL_ROWS, PLA_ALL_COLS, 1, 1,
                                          self.templ, ctypes.byref(h)), "Mscalar_create")
        v = ctypes.c_double(value)
        check(self.lib.PLA_Obj_set(h, MPI_DOUBLE, ctypes.byref(v)), "Obj_set")
        return h

    def free(self, *objs) -> None:
        for o in objs:
            if o is not None and o.value:
                self.lib.PLA_Obj_free(ctypes.byref(o))

    def put(self, obj, a: np.ndarray, i0: int = 0, j0: int = 0) -> None:
        """obj(i0.., j0..) += a through PLA_API_axpy_matrix_to_global."""
        a = np.asfortranarray(a)
        if a.ndim == 1:
            a = a.reshape(-1, 1, order="F")
        one = np.ones(1, dtype=a.dtype)
        check(self.lib.PLA_API_begin(), "API_begin")
        check(self.lib.PLA_Obj_API_open(obj), "API_open")
        check(self.lib.PLA_API_axpy_matrix_to_global(a.shape[0], a.shape[1], one.ctypes.data,
                                                     a.ctypes.data, a.shape[0], obj, i0, j0),
              "axpy_matrix_to_global")
        check(self.lib.PLA_Obj_API_close(obj), "API_close")
        check(self.lib.PLA_API_end(), "API_end")

    def get(self, obj) -> np.ndarray:
        """The object's contents as a column-major numpy array."""
        m, n, dt = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self.lib.PLA_Obj_global_length(obj, ctypes.byref(m))
        self.lib.PLA_Obj_global_width(obj, ctypes.byref(n))
        self.lib.PLA_Obj_datatype(obj, ctypes.byref(dt))
        out = np.zeros((m.value, n.value), dtype=_NP[dt.value], order="F")
        check(self.lib.PLA_Obj_get_local_contents(obj, PLA_NO_TRANSPOSE, None, None,
                                                  out.ctypes.data, max(m.value, 1), 1),
              "get_local_contents")
        return out

    def set(self, obj, a: np.ndarray) -> None:
        a = np.asfortranarray(a)
        if a.ndim == 1:
            a = a.reshape(-1, 1, order="F")
        check(self.lib.PLA_Obj_set_local_contents(PLA_NO_TRANSPOSE, a.shape[0], a.shape[1],
                                                  a.ctypes.data, max(a.shape[0], 1), 1, obj),
              "set_local_contents")

    def close(self) -> None:
        if self.templ.value:
            self.lib.PLA_Temp_free(ctypes.byref(self.templ))
