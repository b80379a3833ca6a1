"""The C-ABI boundary on CPU: librn.so loads, exports every entry point
include/rn.h declares, its structs match the ctypes mirrors field by field,
and without a GPU it refuses to run (no CPU fallback)."""
import ctypes
import os
import re
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "rn.h")


def declared_functions():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(rn_\w+)\s*\(", src, re.M)))


def test_header_declares_the_api():
    names = declared_functions()
    for n in ("rn_create", "rn_destroy", "rn_set_geometry", "rn_set_state", "rn_get_state", "rn_step",
              "rn_read_rect", "rn_request_async", "rn_poll_async", "rn_integrals", "rn_last_error"):
        assert n in names


def test_library_exports_every_declared_symbol(rn):
    from rocket_nozzle_cfd_solver_b200 import solver
    L = solver.lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing
    assert set(declared_functions()) == set(solver.EXPORTS)


def c_layout():
    """sizeof/offsetof of the ABI structs as the C compiler lays them out."""
    prog = r"""
#include <stdio.h>
#include <stddef.h>
#include "rn.h"
#define F(T, m) printf(#T "." #m " %zu\n", offsetof(T, m));
int main(void) {
  printf("rn_params %zu\nrn_read_req %zu\nrn_integral_spec %zu\nrn_integrals_out %zu\n", sizeof(rn_params),
         sizeof(rn_read_req), sizeof(rn_integral_spec), sizeof(rn_integrals_out));
  F(rn_params, amb) F(rn_params, bar) F(rn_params, Tw) F(rn_params, RcCells) F(rn_params, order2)
  F(rn_params, chem) F(rn_params, mhat) F(rn_params, fuel) F(rn_params, ox) F(rn_params, fan)
  F(rn_integral_spec, dx) F(rn_integral_spec, Rs) F(rn_integral_spec, inj) F(rn_integrals_out, t)
  printf("rn_server_opts %zu\nrn_solve_request %zu\nrn_solve_result %zu\nrn_serve_status %zu\n",
         sizeof(rn_server_opts), sizeof(rn_solve_request), sizeof(rn_solve_result), sizeof(rn_serve_status));
  F(rn_server_opts, max_active) F(rn_server_opts, tile) F(rn_server_opts, max_active_cells) F(rn_solve_request, mask) F(rn_solve_request, injTab)
  F(rn_solve_request, P) F(rn_solve_request, spec) F(rn_solve_request, drop) F(rn_solve_request, max_steps)
  F(rn_solve_request, parcelsA) F(rn_solve_request, parcelHead)
  F(rn_solve_result, steps) F(rn_solve_result, done_ms) F(rn_solve_result, integrals) F(rn_serve_status, failed)
  printf("rn_separation_spec %zu\nrn_separation_out %zu\n", sizeof(rn_separation_spec), sizeof(rn_separation_out));
  F(rn_separation_spec, dx) F(rn_separation_spec, pRef) F(rn_separation_out, x) F(rn_separation_out, Msep)
  printf("rn_derived_spec %zu\n", sizeof(rn_derived_spec));
  F(rn_derived_spec, range) F(rn_derived_spec, chemV) F(rn_derived_spec, Tscale) F(rn_derived_spec, dx)
  return 0;
}
"""
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "layout.c")
        exe = os.path.join(d, "layout")
        open(c, "w").write(prog)
        subprocess.run(["gcc", "-I", os.path.dirname(HEADER), c, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    return dict((k, int(v)) for k, v in (line.split() for line in out.strip().splitlines()))


def test_struct_layout_matches_header(rn):
    from rocket_nozzle_cfd_solver_b200 import solver
    c = c_layout()
    assert c["rn_params"] == ctypes.sizeof(solver.RnParams)
    assert c["rn_read_req"] == ctypes.sizeof(solver.RnReadReq)
    assert c["rn_integral_spec"] == ctypes.sizeof(solver.RnIntegralSpec)
    assert c["rn_integrals_out"] == ctypes.sizeof(solver.RnIntegralsOut)
    classes = {"rn_params": solver.RnParams, "rn_integral_spec": solver.RnIntegralSpec,
               "rn_integrals_out": solver.RnIntegralsOut, "rn_server_opts": solver.RnServerOpts,
               "rn_solve_request": solver.RnSolveRequest, "rn_solve_result": solver.RnSolveResult,
               "rn_serve_status": solver.RnServeStatus, "rn_separation_spec": solver.RnSeparationSpec,
               "rn_separation_out": solver.RnSeparationOut, "rn_derived_spec": solver.RnDerivedSpec}
    for t in ("rn_server_opts", "rn_solve_request", "rn_solve_result", "rn_serve_status", "rn_separation_spec",
              "rn_separation_out", "rn_derived_spec"):
        assert c[t] == ctypes.sizeof(classes[t]), t
    for key, v in c.items():
        if "." in key:
            t, m = key.split(".")
            cls = classes[t]
            assert getattr(cls, m).offset == v, key


def has_cuda():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(has_cuda(), reason="checks the behaviour without a CUDA device")
def test_no_cpu_fallback_without_gpu(rn):
    from rocket_nozzle_cfd_solver_b200 import solver
    h = ctypes.c_void_p()
    rc = solver.lib().rn_create(8, 8, ctypes.byref(h))
    assert rc == -2 and not h.value
    assert b"CUDA" in solver.lib().rn_last_error() or b"device" in solver.lib().rn_last_error()
    with pytest.raises(solver.RnError):
        rn.GPUSolver(16, 8)


def test_argument_errors_are_reported(rn):
    from rocket_nozzle_cfd_solver_b200 import solver
    L = solver.lib()
    assert L.rn_create(8, 8, None) == -1
    assert b"NULL" in L.rn_last_error()
    assert L.rn_step(None, 1, None) == -1
    assert L.rn_destroy(None) == 0


def test_oracle_library_exports():
    import __graft_entry__ as ge
    o = ge.load_oracle()
    L = o.lib()
    src = open(os.path.join(ROOT, "oracle", "rn_oracle.h")).read()
    for n in re.findall(r"^\s*(?:void\*?|int)\s+(rno_\w+)\s*\(", src, re.M):
        assert hasattr(L, n), n
