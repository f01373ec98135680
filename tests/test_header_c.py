"""The boundary as a C or C++ caller meets it: include/abm_capi.h compiles as strict C99 and
as C++17 with every warning an error, a program that names every declared entry point links
against the shipped library, and, run without a GPU, abm_create fails with ABM_ERR_CUDA and a
readable reason that the returned context carries until abm_destroy.  Host compilers only,
no device code runs."""
import os
import shutil
import subprocess

import pytest

import abm_b200
from test_capi_cpu import ROOT, header_functions

PROGRAM = r"""
#include <stdio.h>
#include <string.h>
#include "abm_capi.h"

/* every entry point the header declares, so the link fails if the library lacks one */
static void (*const entry_points[])(void) = {
%(entries)s
};

int main(void)
{
    abm_params p;
    abm_ctx* ctx = NULL;
    int rc;
    memset(&p, 0, sizeof(p));
    p.R = 0.8; p.Rcell = 0.5; p.E0 = 3900.0; p.Ecell = 3.9e6; p.L0 = 2.0; p.Ldiv = 5.6;
    p.neighbor_threshold = 3.6; p.integration_mode = ABM_DORMAND_PRINCE; p.max_stepsize = 1e-5;
    p.max_error_allowed = 1e-8; p.iter_update_stepsize = 1; p.iter_update_neighbors = 1;
    p.cap_cells = 64;
    if (abm_create(NULL, &ctx) != ABM_ERR_ARG) return 10;      /* a NULL argument: no context */
    rc = abm_create(&p, &ctx);
    printf("%%d|%%s|%%d\n", rc, ctx ? abm_last_error(ctx) : "", (int)(sizeof(entry_points) / sizeof(entry_points[0])));
    if (ctx) abm_destroy(ctx);
    return 0;
}
"""


def build_and_run(tmp_path, compiler, std_flags, suffix):
    names = header_functions()
    src = tmp_path / ("caller" + suffix)
    src.write_text(PROGRAM % {"entries": ",\n".join("    (void (*)(void))%s" % n for n in names)})
    exe = tmp_path / ("caller_" + compiler.replace("+", "p"))
    libdir = os.path.dirname(abm_b200.LIB_PATH)
    cmd = [compiler] + std_flags + ["-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
                                    str(src), "-o", str(exe), "-L", libdir, "-labm_b200",
                                    "-Wl,-rpath," + libdir]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.strip()
    rc, msg, count = out.split("|")
    return int(rc), msg, int(count), len(names)


@pytest.mark.parametrize("compiler, flags, suffix", [
    ("gcc", ["-std=c99", "-pedantic"], ".c"),
    ("g++", ["-std=c++17", "-pedantic"], ".cpp"),
])
def test_header_compiles_links_and_reports(tmp_path, compiler, flags, suffix):
    if shutil.which(compiler) is None:
        pytest.skip("%s not installed" % compiler)
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except ImportError:
        has_gpu = False
    rc, msg, count, declared = build_and_run(tmp_path, compiler, flags, suffix)
    assert count == declared
    if has_gpu:
        assert rc == 0
    else:
        assert rc == -2 and msg.startswith("no CUDA device"), (rc, msg)
