"""The public header is plain C: a C99 program that includes include/fastcone_b200.h
compiles with gcc -Wall -Werror -pedantic, links against the library, and calls a
reference entry point the way a C caller of wrapper.c would (the reference's own wrapper.h
does not compile: it declares pixelWidth twice, wrapper.h:49-109).  The call uses a device
index that does not exist, so it runs without a GPU: the void entry point must return and
leave FCB_ERR_NODEVICE in fcb_last_status() instead of exiting the process."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROGRAM = r"""
#include <stdio.h>
#include "fastcone_b200.h"

int main(void)
{
  float vol[8] = {0}, proj[2 * 4 * 4] = {0}, angles[2] = {0.0f, 1.0f}, hmid[2] = {1.0f, 1.0f};
  float norm[2] = {0.5f, 0.5f};
  int volDim[3] = {2, 2, 2}, volStart[3] = {0, 0, 0}, volEnd[3] = {2, 2, 2};
  int projDim[3] = {4, 4, 2}, projWH[2] = {4, 4}, woff[2] = {0, 0}, hoff[2] = {0, 0};
  if (fcb_version() < 10000) return 2;
  GPU_CB_K_backproject(9999, vol, proj, angles, hmid, 50.0f, 1.0f, volDim, volStart, volEnd, projDim,
                       projWH, woff, hoff, norm, 2);
  printf("%d %s\n", fcb_last_status(), fcb_last_error());
  return fcb_last_status() == FCB_ERR_NODEVICE ? 0 : 1;
}
"""


def test_header_compiles_as_c_and_reference_entry_point_reports_status():
    if shutil.which("gcc") is None:
        pytest.skip("gcc not available")
    libdir = os.path.join(ROOT, "fastcone_b200")
    if not os.path.exists(os.path.join(libdir, "libfastcone_b200.so")):
        pytest.skip("library not built")
    out = os.path.join(libdir, "_build", "c_caller")  # git-ignored build folder
    os.makedirs(out, exist_ok=True)
    src = os.path.join(out, "caller.c")
    exe = os.path.join(out, "caller")
    with open(src, "w") as f:
        f.write(PROGRAM)
    cc = subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic",
                         "-I", os.path.join(ROOT, "include"), src, "-L", libdir, "-lfastcone_b200",
                         "-Wl,-rpath," + libdir, "-o", exe], capture_output=True, text=True)
    assert cc.returncode == 0, cc.stderr
    run = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert run.returncode == 0, (run.stdout, run.stderr)
