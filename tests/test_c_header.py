"""The boundary headers are plain C (what a cgo / JNI / N-API binding
includes): a C99 program compiled with gcc against `include/*.h` links the
native library and gets the documented host-side error codes, no GPU
needed."""
import shutil
import subprocess

import pytest

from tests.conftest import ROOT

C_PROGRAM = r"""
#include <stdio.h>
#include <string.h>
#include "fbalp.h"
#include "fbalp_mlp.h"

int main(void) {
    int bad = 0;
    if (fbalp_engine_destroy(NULL) != FBALP_ERR_INVALID) bad |= 1;
    const char* msg = fbalp_last_error();
    if (msg == NULL || strlen(msg) == 0) bad |= 2;
    fbalp_options opt;
    fbalp_default_options(&opt);
    if (opt.warps_per_block != 16) bad |= 4;
    fbalp_solve_params prm;
    fbalp_default_solve_params(&prm);
    if (prm.check_every != 64) bad |= 8;
    /* invalid GEMM: K = 0 */
    if (fbalp_gemm_bf16(4, 4, 0, (void*)16, 8, 0, (void*)16, 8, 0, NULL, FBALP_EPI_NONE, 1.0f,
                        (float*)16, NULL, 4, NULL, 0, 0, NULL) != FBALP_MLP_ERR_INVALID) bad |= 16;
    /* invalid certificate: neq > rows */
    if (fbalp_scaled_certificate(0, 2, 3, 3, NULL, NULL, NULL, NULL, NULL, NULL, 0, NULL, NULL, NULL, NULL, NULL,
                                 NULL, NULL, NULL, NULL, NULL, NULL, 1, NULL, NULL, NULL, NULL, NULL)
        != FBALP_ERR_INVALID) bad |= 32;
    printf("%d\n", bad);
    return bad;
}
"""


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc needed")
def test_headers_compile_as_c99_and_link(native_built, tmp_path):
    src = tmp_path / "boundary.c"
    src.write_text(C_PROGRAM)
    exe = tmp_path / "boundary"
    lib = native_built
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-pedantic", "-I", str(ROOT / "include"), str(src),
                    "-L", str(lib.parent), "-lfbalp", f"-Wl,-rpath,{lib.parent}", "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
