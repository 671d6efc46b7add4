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


# ---- callers that bring their own MPI ---------------------------------------
# A reference driver includes <mpi.h> and then PLA.h (or only PLA.h, which in
# the reference includes <mpi.h> itself: INCLUDE/PLA.h:14) and passes its MPI's
# own handles.  The two stand-in MPI headers under tests/abi/ have MPICH-style
# int handles and Open-MPI-style pointer handles, none equal to the library's
# codes; the header translates them at each call.

MPI_HOST_DRIVER = r"""
#include <stdio.h>
#include <string.h>
#include <sys/stat.h>
%(first)s
#include "PLA.h"

int main(int argc, char **argv) {
  MPI_Comm comm = MPI_COMM_NULL;
  PLA_Mixed_params p;
  struct stat st;
  int fd = -1, i;
  char name[512];
  static const struct { const char *what; int bytes; } cases[] = {
      {"double", 8}, {"float", 4}, {"int", 4}};
  MPI_Datatype dts[3];
  dts[0] = MPI_DOUBLE;
  dts[1] = MPI_FLOAT;
  dts[2] = MPI_INT;
  MPI_Init(&argc, &argv);
  if (argc < 2) return 10;
  /* TEST/test_lu.c's mesh call on a 1 x 1 mesh: a communicator comes back */
  if (PLA_Comm_1D_to_2D(MPI_COMM_WORLD, 1, 1, &comm) != PLA_SUCCESS) return 11;
  if (comm == MPI_COMM_NULL) return 12;
  if (PLA_Comm_1D_to_2D(MPI_COMM_WORLD, 2, 1, &comm) == PLA_SUCCESS) return 13;
  PLA_Clear_error();
  /* the caller's datatype handles size the library's files */
  for (i = 0; i < 3; i++) {
    snprintf(name, sizeof name, "%%s/f%%d.bin", argv[1], i);
    if (PLA_File_create(name, dts[i], 100, &fd) != PLA_SUCCESS) return 20 + i;
    PLA_File_close(fd);
    if (stat(name, &st) != 0 || st.st_size != 100 * cases[i].bytes) return 30 + i;
    PLA_File_unlink(name);
  }
  /* a handle the library does not take is an error, not a guess */
  snprintf(name, sizeof name, "%%s/bad.bin", argv[1]);
  if (PLA_File_create(name, MPI_LONG, 100, &fd) != PLA_ERROR) return 40;
  PLA_Clear_error();
  PLA_Mixed_params_default(&p);
  if (p.precision != PLA_B200_PREC_FP16) return 41;
  MPI_Finalize();
  printf("ok\n");
  return 0;
}
"""

MPI_SOLVE_DRIVER = r"""
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <mpi.h>
#include "PLA.h"

/* a reference-style driver: mesh, PLA_Init, template, objects created with
   the caller's MPI datatypes, fill through the API, PLA_General_solve */
int main(int argc, char **argv) {
  int n = 200, i, j, nb = 64;
  MPI_Comm comm = MPI_COMM_NULL;
  MPI_Datatype dt = MPI_DATATYPE_NULL;
  PLA_Template templ = NULL;
  PLA_Obj A = NULL, piv = NULL, b = NULL;
  double one = 1.0, err = 0.0, *a = malloc(sizeof(double) * n * n), *x = malloc(sizeof(double) * n);
  MPI_Init(&argc, &argv);
  if (PLA_Comm_1D_to_2D(MPI_COMM_WORLD, 1, 1, &comm)) return 1;
  if (PLA_Init(comm)) return 2;
  pla_Environ_set_nb_alg(PLA_OP_ALL_ALG, nb);
  if (PLA_Temp_create(nb, 0, &templ)) return 3;
  if (PLA_Matrix_create(MPI_DOUBLE, n, n, templ, PLA_ALIGN_FIRST, PLA_ALIGN_FIRST, &A)) return 4;
  if (PLA_Mvector_create(MPI_INT, n, 1, templ, PLA_ALIGN_FIRST, &piv)) return 5;
  if (PLA_Mvector_create(MPI_DOUBLE, n, 1, templ, PLA_ALIGN_FIRST, &b)) return 6;
  if (PLA_Obj_datatype(A, &dt) || dt != MPI_DOUBLE) return 7;
  if (PLA_Obj_datatype(piv, &dt) || dt != MPI_INT) return 8;
  srand48(5);
  for (j = 0; j < n; j++)
    for (i = 0; i < n; i++) a[i + (size_t)j * n] = drand48() * 2 - 1 + (i == j ? 4.0 : 0.0);
  for (i = 0; i < n; i++) {          /* b = A * ones */
    x[i] = 0.0;
    for (j = 0; j < n; j++) x[i] += a[i + (size_t)j * n];
  }
  PLA_API_begin();
  PLA_Obj_API_open(A);
  PLA_Obj_API_open(b);
  PLA_API_axpy_matrix_to_global(n, n, &one, a, n, A, 0, 0);
  PLA_API_axpy_vector_to_global(n, &one, x, 1, b, 0);
  PLA_Obj_API_close(A);
  PLA_Obj_API_close(b);
  PLA_API_end();
  if (PLA_General_solve(A, piv, b)) return 9;
  if (PLA_Obj_get_local_contents(b, PLA_NO_TRANSPOSE, NULL, NULL, x, n, 1)) return 10;
  for (i = 0; i < n; i++) err = fmax(err, fabs(x[i] - 1.0));
  PLA_Obj_free(&A);
  PLA_Obj_free(&piv);
  PLA_Obj_free(&b);
  PLA_Temp_free(&templ);
  PLA_Finalize();
  MPI_Comm_free(&comm);
  MPI_Finalize();
  printf("err %.3e\n", err);
  return err < 1e-10 ? 0 : 11;
}
"""


def _compile(tmp_path, src_text, mpi_dir, name, extra=()):
    import shutil
    import subprocess
    if not shutil.which("cc"):
        pytest.skip("no cc")
    src = tmp_path / f"{name}.c"
    src.write_text(src_text)
    exe = tmp_path / name
    libdir = os.path.dirname(LIB)
    cmd = ["cc", "-std=c99", "-D_DEFAULT_SOURCE", "-Wall", "-Werror", "-o", str(exe), str(src),
           "-I", os.path.join(ROOT, "tests", "abi", mpi_dir), "-I", os.path.join(ROOT, "include"),
           "-L", libdir, "-lplapack_b200", f"-Wl,-rpath,{libdir}", "-lm", *extra]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


@pytest.mark.parametrize("mpi_dir", ["mpich_like", "ompi_like"])
@pytest.mark.parametrize("first", ["#include <mpi.h>", ""])
def test_driver_with_its_own_mpi_handles(built_lib, tmp_path, mpi_dir, first):
    """Host-only calls with the caller's MPI handles: the 1 x 1 mesh call, and
    files sized by the caller's datatypes (PLA_File_create takes a datatype
    and needs no GPU).  With `first` empty the driver includes only PLA.h,
    which finds <mpi.h> on the include path as the reference's header does."""
    import subprocess
    exe = _compile(tmp_path, MPI_HOST_DRIVER % {"first": first}, mpi_dir, "host_driver")
    r = subprocess.run([str(exe), str(tmp_path)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and r.stdout.startswith("ok"), (r.returncode, r.stdout, r.stderr)


def test_without_mpi_the_names_are_the_codes(built_lib, tmp_path):
    import subprocess
    src = r"""
#include "PLA.h"
int main(void) {
  return (MPI_DOUBLE == PLA_B200_DT_DOUBLE && MPI_INT == PLA_B200_DT_INT &&
          MPI_COMM_WORLD == PLA_B200_COMM_WORLD && sizeof(MPI_Datatype) == sizeof(int)) ? 0 : 1;
}
"""
    exe = _compile(tmp_path, src, "no_such_dir", "plain", extra=["-DPLA_B200_NO_MPI"])
    assert subprocess.run([str(exe)], timeout=60).returncode == 0


@pytest.mark.gpu
@pytest.mark.parametrize("mpi_dir", ["mpich_like", "ompi_like"])
def test_reference_style_solve_with_its_own_mpi(built_lib, tmp_path, mpi_dir):
    """A 200 x 200 PLA_General_solve from a C driver that created its objects
    with its own MPI's MPI_DOUBLE / MPI_INT handles."""
    import subprocess
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    exe = _compile(tmp_path, MPI_SOLVE_DRIVER, mpi_dir, "solve_driver")
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.startswith("err"), (r.returncode, r.stdout, r.stderr)
