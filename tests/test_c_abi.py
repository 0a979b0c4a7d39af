"""The C-ABI from plain C: include/ccsd_b200.h compiles as C11 with warnings as errors, and a
C program drives the library on a planning-only context (no device): spaces, tensors, one
contraction statement and its flop count, the CCSD and Lambda plan queries, the DIIS entry
points' argument checks, error codes and messages.  This is the binding surface a cgo / JNI / ctypes caller sees."""
import os
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
PROGRAM = r"""
#include <stdio.h>
#include <string.h>
#include "ccsd_b200.h"

#define CHECK(x) do { int st_ = (x); if (st_) { fprintf(stderr, "%s -> %d\n", #x, st_); return 1; } } while (0)

int main(void) {
    ccsd_ctx ctx = NULL;
    CHECK(ccsd_ctx_create(-1, NULL, &ctx));                  /* planning only */
    int vrt[1] = {6}, occ[1] = {2};
    CHECK(ccsd_ctx_set_spaces(ctx, 1, vrt, NULL, occ, NULL));   /* closed shell */
    if (ccsd_ctx_set_spaces(ctx, 1, NULL, NULL, occ, NULL) != CCSD_ERR_ARG) return 1;
    int vv_oo[2] = {2, 0}, oo_vv[2] = {0, 2}, none[2] = {0, 0};
    ccsd_tensor V, T, Z;
    CHECK(ccsd_tensor_create(ctx, "V", vv_oo, vv_oo, 0, &V));   /* <ab||cd>: nout {2,0}, nin {2,0} */
    CHECK(ccsd_tensor_create(ctx, "T", vv_oo, oo_vv, 0, &T));
    CHECK(ccsd_tensor_create(ctx, "Z", vv_oo, oo_vv, 0, &Z));
    CHECK(ccsd_contract(ctx, 0.5, V, "abef", T, "efij", 1.0, Z, "abij"));
    double flops = 0;
    CHECK(ccsd_ctx_plan_flops(ctx, &flops));
    /* 4 C(6,2)^2 C(2,2) + 2 * 6^4 * 2^2 */
    if (flops != 4.0 * 15 * 15 * 1 + 2.0 * 1296 * 4) { fprintf(stderr, "flops %g\n", flops); return 1; }
    /* a bad index string is an error with a message, not a crash */
    int st = ccsd_contract(ctx, 1.0, V, "abex", T, "efij", 1.0, Z, "abij");
    if (st == 0 || strlen(ccsd_last_error(ctx)) == 0) { fprintf(stderr, "bad statement accepted\n"); return 1; }
    /* reading data from a planning context is refused */
    double x;
    int alpha[4] = {2, 0, 0, 2}, irr[4] = {0, 0, 0, 0};
    if (ccsd_tensor_read_block(ctx, T, alpha, irr, &x) != CCSD_ERR_UNSUPPORTED) return 1;
    /* NULL where the ABI writes a result is an argument error, not a crash */
    int64_t nb;
    int nd;
    if (ccsd_ctx_device_bytes(ctx, NULL) != CCSD_ERR_ARG) return 1;
    if (ccsd_tensor_ndim(ctx, T, NULL) != CCSD_ERR_ARG) return 1;
    if (ccsd_tensor_block_size(ctx, T, NULL, irr, &nb) != CCSD_ERR_ARG) return 1;
    if (ccsd_tensor_create(ctx, "X", NULL, oo_vv, 0, &Z) != CCSD_ERR_ARG) return 1;
    if (ccsd_ctx_plan_flops(ctx, NULL) != CCSD_ERR_ARG) return 1;
    CHECK(ccsd_tensor_ndim(ctx, T, &nd));
    CHECK(ccsd_tensor_block_size(ctx, T, alpha, irr, &nb));
    if (nd != 4 || nb != 6 * 6 * 2 * 2) return 1;
    (void)none;
    /* DIIS over caller tensors needs tensors with data: refused on a planning context;
       NULL handles and outputs are argument errors */
    ccsd_diis d = NULL;
    if (ccsd_diis_create(ctx, 8, 1, 0.0, &d) != CCSD_ERR_UNSUPPORTED || d != NULL) return 1;
    if (ccsd_diis_create(ctx, 8, 1, 0.0, NULL) != CCSD_ERR_ARG) return 1;
    if (ccsd_diis_extrapolate(NULL, 1, &T, &Z, NULL) != CCSD_ERR_ARG) return 1;
    if (ccsd_diis_coefficients(NULL, &nd, NULL) != CCSD_ERR_ARG) return 1;
    if (ccsd_diis_destroy(NULL) != CCSD_ERR_ARG) return 1;
    CHECK(ccsd_ctx_destroy(ctx));

    ccsd_options o;
    ccsd_options_default(&o);
    double f_iter = 0, f_hbar = 0, f_lam = 0;
    int64_t bytes = 0, lbytes = 0;
    CHECK(ccsd_plan_query(1, vrt, occ, &o, 1, &f_iter, &bytes));
    CHECK(ccsd_lambda_plan_query(1, vrt, occ, &o, &f_hbar, &f_lam, &lbytes));
    if (!(f_iter > 0 && bytes > 0 && f_hbar > 0 && f_lam > 0 && lbytes > 0)) return 1;
    printf("ok %g %g %g\n", f_iter, f_hbar, f_lam);
    return 0;
}
"""


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_header_is_c11_and_drives_a_planning_context(built_lib, tmp_path):
    src = tmp_path / "abi.c"
    src.write_text(PROGRAM)
    exe = tmp_path / "abi"
    lib_dir = ROOT / "aquarius_b200"
    cmd = ["gcc", "-std=c11", "-Wall", "-Wextra", "-Werror", "-pedantic", "-I", str(ROOT / "include"), str(src),
           "-o", str(exe), "-L", str(lib_dir), "-lccsd_b200", f"-Wl,-rpath,{lib_dir}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    env = dict(os.environ)
    env["LD_LIBRARY_PATH"] = ":".join(filter(None, ["/usr/local/cuda/lib64", env.get("LD_LIBRARY_PATH")]))
    r = subprocess.run([str(exe)], capture_output=True, text=True, env=env, timeout=120)
    assert r.returncode == 0 and r.stdout.startswith("ok"), r.stdout + r.stderr
