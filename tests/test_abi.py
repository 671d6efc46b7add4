"""The C-ABI library builds, loads and exports every function include/*.h declares.

No GPU is needed: only symbol resolution is checked, nothing is computed.
"""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "plapack_b200", "libplapack_b200.so")


def declared_functions():
    names = set()
    for h in ("PLA.h", "pla_b200.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:int\s+|void\s*\*\s*|void\s+)(\w+)\s*\(", text,
                             flags=re.M):
            names.add(m.group(1))
    return sorted(names)


@pytest.fixture(scope="module")
def built_lib():
    if not os.path.exists(LIB):
        from plapack_b200 import build
        build.build()
    return ctypes.CDLL(LIB)


def test_header_declares_the_reference_surface():
    names = set(declared_functions())
    for need in ["PLA_Init", "PLA_Temp_create", "PLA_Matrix_create", "PLA_Mvector_create",
                 "PLA_Obj_view", "PLA_Obj_split_4", "PLA_API_axpy_matrix_to_global", "PLA_LU",
                 "PLA_Chol", "PLA_Trsm", "PLA_Gemm", "PLA_Trsv", "PLA_General_solve",
                 "PLA_Pos_def_solve", "PLA_Local_gemm", "PLA_Local_trsm", "PLA_Local_syrk",
                 "PLA_Local_iamax", "PLA_Local_ger", "PLA_Local_inv_scal"]:
        assert need in names, need


def test_every_declared_symbol_is_exported(built_lib):
    missing = [n for n in declared_functions() if not hasattr(built_lib, n)]
    assert not missing, missing


def test_binding_loads(built_lib):
    from plapack_b200 import pla
    lib = pla.load()
    assert lib.PLA_LU.restype is ctypes.c_int


def test_header_declares_what_the_reference_drivers_call():
    # the PLA_* calls of TEST/test_lu.c, TEST/test_chol.c, the EXAMPLES drivers
    # and SOLVERS/LINPACK/driver.c outside the out-of-core family
    names = set(declared_functions())
    for need in ["PLA_Axpy", "PLA_Nrm2", "PLA_Shift", "PLA_malloc", "PLA_calloc", "PLA_free",
                 "PLA_LU_linpack", "PLA_LU_linpack_right", "PLA_Copy", "PLA_Iamax",
                 "PLA_Obj_get_local_contents", "PLA_Create_constants_conf_to"]:
        assert need in names, need


def test_host_memory_helpers(built_lib):
    # OBJ/PLA_Memory.c: malloc / calloc with running totals; host memory only
    from plapack_b200 import pla
    lib = pla.load()
    base = lib.PLA_Total_size_malloced()
    p = lib.PLA_malloc(1000)
    q = lib.PLA_calloc(250, 8)
    assert p and q
    assert lib.PLA_Total_size_malloced() == base + 3000
    assert lib.PLA_Max_size_malloced() >= base + 3000
    assert bytes((ctypes.c_char * 2000).from_address(q)) == b"\0" * 2000
    ctypes.memset(p, 7, 1000)                      # the whole block is usable
    assert lib.PLA_free(p) is None
    assert lib.PLA_free(q) is None
    assert lib.PLA_free(None) is None              # freeing NULL is a no-op
    assert lib.PLA_Total_size_malloced() == base


def test_file_layer_without_gpu(built_lib, tmp_path):
    # IO/PLA_File.c: create (sized), close, open again, unlink; IO/PLA_File_stats.c counters
    from plapack_b200 import pla
    lib = pla.load()
    name = str(tmp_path / "ooc.bin").encode()
    fd = ctypes.c_int(-1)
    assert lib.PLA_File_create(name, pla.MPI_DOUBLE, 1000, ctypes.byref(fd)) == 0
    assert fd.value >= 0
    assert os.path.getsize(name) == 8000
    assert lib.PLA_File_close(fd.value) == 0
    assert lib.PLA_File_open(name, pla.MPI_DOUBLE, 1000, ctypes.byref(fd)) == 0
    assert lib.PLA_File_close(fd.value) == 0
    assert lib.PLA_File_unlink(name) == 0
    assert not os.path.exists(name)
    assert lib.PLA_File_open(name, pla.MPI_DOUBLE, 1000, ctypes.byref(fd)) == pla.PLA_ERROR
    assert lib.PLA_File_stats_start() == 0
    v = [ctypes.c_double(-1) for _ in range(4)]
    assert lib.PLA_B200_file_stats(*[ctypes.byref(x) for x in v]) == 0
    assert [x.value for x in v] == [0.0, 0.0, 0.0, 0.0]


C_DRIVER = r"""
#include <stdio.h>
#include <string.h>
#include "PLA.h"
#include "pla_b200.h"

/* every solver entry point a PLAPACK driver calls, by address: the link
   resolves them all against the library */
static void *const entry_points[] = {
  (void *)PLA_Init, (void *)PLA_Finalize, (void *)PLA_Temp_create, (void *)PLA_Matrix_create,
  (void *)PLA_Mvector_create, (void *)PLA_API_axpy_matrix_to_global, (void *)PLA_LU,
  (void *)PLA_Chol, (void *)PLA_Trsv, (void *)PLA_Trsm, (void *)PLA_Gemm,
  (void *)PLA_General_solve, (void *)PLA_Pos_def_solve, (void *)PLA_General_solve_mixed,
  (void *)PLA_OOC_Chol, (void *)PLA_Batch_plan_create};

int main(void) {
  PLA_Mixed_params p;
  void *m;
  size_t i;
  for (i = 0; i < sizeof entry_points / sizeof entry_points[0]; i++)
    if (!entry_points[i]) return 1;
  memset(&p, 0xff, sizeof p);
  PLA_Mixed_params_default(&p);   /* host only: fills the defaults */
  if (p.precision != PLA_B200_PREC_FP16 || p.refinement != PLA_B200_IR_GMRES || !p.escalate)
    return 2;
  m = PLA_malloc(64);             /* host memory, no device needed */
  if (!m || PLA_free(m) != NULL) return 3;
  printf("ok %d %d\n", PLA_SUCCESS, PLA_LOWER_TRIANGULAR);
  return 0;
}
"""


@pytest.mark.parametrize("compiler,std", [("cc", "-std=c99"), ("c++", "-std=c++17")])
def test_c_driver_compiles_links_and_runs(built_lib, tmp_path, compiler, std):
    """The header is plain C (and C++ through its extern "C" guard), and the
    link line of the integration guide resolves a driver's entry points."""
    import shutil
    import subprocess
    if not shutil.which(compiler):
        pytest.skip(f"no {compiler}")
    src = tmp_path / ("driver.c" if compiler == "cc" else "driver.cpp")
    src.write_text(C_DRIVER)
    exe = tmp_path / "driver"
    libdir = os.path.dirname(LIB)
    cmd = [compiler, std, "-Wall", "-Werror", "-o", str(exe), str(src),
           "-I", os.path.join(ROOT, "include"), "-L", libdir, "-lplapack_b200",
           f"-Wl,-rpath,{libdir}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and r.stdout.startswith("ok 0 52"), (r.returncode, r.stdout, r.stderr)
