"""include/dglm.h is a plain C interface: a C99 and a C++11 program include
it, link libdglm.so and call entry points that need no GPU (version, order
table, argument validation)."""
import os
import shutil
import subprocess

import pytest

from exadglm_b200 import build as _build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "exadglm_b200", "libdglm.so")

PROGRAM = r"""
#include <stdio.h>
#include <string.h>
#include "dglm.h"

int main(void) {
  dglm_desc d;
  dglm_handle *h = 0;
  double t = 0.0, dt = 0.0;
  int tstep = 0, bad = 7, ok;
  memset(&d, 0, sizeof d);
  ok = dglm_abi_version() == DGLM_ABI_VERSION;
  ok = ok && dglm_order_supported(4) == 1 && dglm_order_supported(99) == 0;
  ok = ok && dglm_create(0, &h) == DGLM_ERR_INVALID;
  ok = ok && dglm_create(&d, 0) == DGLM_ERR_INVALID;
  ok = ok && dglm_step(0, 1) == DGLM_ERR_INVALID;
  ok = ok && dglm_get_time(0, &t, &dt, &tstep) == DGLM_ERR_INVALID;
  ok = ok && dglm_set_time(0, 1.0, 1) == DGLM_ERR_INVALID;
  ok = ok && dglm_run_ensemble(0, 1, 0, 0, 1, &bad) == DGLM_ERR_INVALID && bad == -1;
  ok = ok && dglm_last_error() != 0 && dglm_last_error()[0] != 0;
  ok = ok && dglm_destroy(0) == DGLM_OK;
  printf("%s\n", ok ? "c-abi ok" : "c-abi FAILED");
  return ok ? 0 : 1;
}
"""


@pytest.mark.parametrize("compiler,std,src", [("gcc", "-std=c99", "prog.c"),
                                              ("g++", "-std=c++11", "prog.cpp")])
def test_header_compiles_links_and_runs(tmp_path, compiler, std, src):
    if not os.path.exists(LIB):
        pytest.skip("libdglm.so not built")
    if shutil.which(compiler) is None:
        pytest.skip(f"{compiler} not found")
    path = tmp_path / src
    path.write_text(PROGRAM)
    exe = str(tmp_path / "prog")
    r = subprocess.run([compiler, std, "-Wall", "-Wextra", "-pedantic", "-Werror",
                        "-I", _build.INCLUDE, str(path), "-o", exe,
                        "-L", os.path.dirname(LIB), "-ldglm",
                        "-Wl,-rpath," + os.path.dirname(LIB)],
                       stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    assert r.returncode == 0, r.stdout
    r = subprocess.run([exe], stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True,
                       timeout=60)
    assert r.returncode == 0 and "c-abi ok" in r.stdout, r.stdout
