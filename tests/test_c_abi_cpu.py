"""The C ABI from C and C++ callers, without a GPU: include/pimc_b200.h
compiles as C99 and as C++17 with warnings as errors, a C program links
against libpimc_b200.so and gets from the host-only entry points the
values the Python layer gets, and pimc_create on a machine without a
usable device returns a status code instead of crashing."""
import os
import shutil
import subprocess

import numpy as np
import pytest

import pimcplusplus_b200 as P
from helpers import ROOT, lj_case
from pimcplusplus_b200 import workloads as W

LIBDIR = os.path.join(ROOT, "pimcplusplus_b200")
INCLUDE = os.path.join(ROOT, "include")

PROGRAM = r"""
#include <stdio.h>
#include "pimc_b200.h"

int main(int argc, char **argv) {
  double u = 0.0, box[3] = {9.0, 10.0, 11.0}, pos[4 * 3];
  int ng, nc, nt, tp, gt, rc, i;
  double g0, g1;
  pimc_system_desc d;
  pimc_context *ctx = 0;
  int species[4] = {0, 0, 0, 0};
  double lam[1] = {6.0596};
  printf("version %d\n", pimc_version());
  printf("status %s\n", pimc_status_string(PIMC_E_ARG));
  rc = pimc_stream_uniform(5ull, 3u, 7ull, &u);
  printf("uniform %d %.17g\n", rc, u);
  rc = pimc_init_random_fixed(box, 4, 0.5, 11ull, pos);
  printf("init %d", rc);
  for (i = 0; i < 12; i++) printf(" %.17g", pos[i]);
  printf("\n");
  rc = pimc_dm_read_info(argv[1], atof_tau(argv[2]), &ng, &nc, &nt, &tp, &gt, &g0, &g1);
  printf("dm %d %d %d %d %d %d %.17g %.17g\n", rc, ng, nc, nt, tp, gt, g0, g1);
  d.num_particles = 4; d.num_time_slices = 5; d.box[0] = 9.0; d.box[1] = 10.0; d.box[2] = 11.0;
  d.tau = 0.01; d.num_species = 1; d.species_of = species; d.lambda = lam; d.num_images = 0; d.device = 0;
  rc = pimc_create(&d, &ctx);
  printf("create %d\n", rc);
  if (rc == PIMC_OK) pimc_destroy(ctx);
  rc = pimc_init_random_fixed(box, 4, -1.0, 11ull, pos);
  printf("badarg %d\n", rc);
  return 0;
}
"""


def _compiler(name):
    path = shutil.which(name)
    if path is None:
        pytest.skip(f"{name} not found")
    return path


def test_header_compiles_as_c_and_cxx(tmp_path):
    src_c = tmp_path / "h.c"
    src_c.write_text('#include "pimc_b200.h"\nint main(void) { return pimc_version() > 0 ? 0 : 1; }\n')
    subprocess.run([_compiler("gcc"), "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic", "-I", INCLUDE, "-c",
                    str(src_c), "-o", str(tmp_path / "h.o")], check=True)
    src_cc = tmp_path / "h.cc"
    src_cc.write_text('#include "pimc_b200.h"\nint main() { pimc_context *c = nullptr; (void)c; return 0; }\n')
    subprocess.run([_compiler("g++"), "-std=c++17", "-Wall", "-Wextra", "-Werror", "-I", INCLUDE, "-c",
                    str(src_cc), "-o", str(tmp_path / "hh.o")], check=True)


def test_c_program_calls_host_entry_points(tmp_path):
    cfg, tau, box, dm = lj_case(tmp_path, n=16, m=16, levels=2, npts=200)
    src = tmp_path / "prog.c"
    src.write_text("#include <stdlib.h>\nstatic double atof_tau(const char *s) { return strtod(s, 0); }\n" + PROGRAM)
    exe = tmp_path / "prog"
    subprocess.run([_compiler("gcc"), "-std=c99", "-Wall", "-Werror", "-I", INCLUDE, str(src), "-o", str(exe),
                    "-L", LIBDIR, "-lpimc_b200", f"-Wl,-rpath,{LIBDIR}"], check=True)
    out = subprocess.run([str(exe), dm, repr(tau)], capture_output=True, text=True, timeout=120, check=True).stdout
    lines = dict(line.split(" ", 1) for line in out.strip().splitlines())
    assert int(lines["version"]) == P.lib().pimc_version()
    assert lines["status"] == P.lib().pimc_status_string(P.PIMC_E_ARG).decode()
    rc, u = lines["uniform"].split()
    assert rc == "0" and float(u) == P.stream_uniform(5, 3, 7)
    vals = lines["init"].split()
    assert vals[0] == "0"
    want = P.init_random_fixed(np.array([9.0, 10.0, 11.0]), 4, 0.5, 11)
    assert np.array_equal(np.array([float(x) for x in vals[1:]]).reshape(4, 3), want)
    dmv = lines["dm"].split()
    t = P.read_dm(dm, tau)
    assert dmv[0] == "0" and [int(x) for x in dmv[1:6]] == [t["num_grid"], t["num_cols"], t["num_tau"],
                                                              t["tau_pos"], t["grid_type"]]
    assert float(dmv[6]) == t["grid_start"] and float(dmv[7]) == t["grid_end"]
    assert int(lines["create"]) in (P.PIMC_OK, 2)  # PIMC_E_CUDA where no device can be used
    assert int(lines["badarg"]) == P.PIMC_E_ARG
