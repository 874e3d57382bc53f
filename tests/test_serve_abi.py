"""CPU tests of the serving ABI: the ctypes structures of the Python
front-end have the layout the C header gives fq_request, fq_result and
fq_server_counters (checked by compiling a probe with the system C
compiler), and a server cannot be created where no device is present."""
import ctypes
import os
import shutil
import subprocess

import pytest

from conftest import ROOT

PROBE = r"""
#include <stddef.h>
#include <stdio.h>
#include "forqaoa.h"
#define F(T, m) printf(#T "." #m " %zu\n", offsetof(T, m));
int main(void) {
    printf("fq_request %zu\nfq_result %zu\nfq_server_counters %zu\n", sizeof(fq_request),
           sizeof(fq_result), sizeof(fq_server_counters));
    F(fq_request, session) F(fq_request, N) F(fq_request, P) F(fq_request, graph_upper)
    F(fq_request, gammas) F(fq_request, betas)
    F(fq_result, ticket) F(fq_result, session) F(fq_result, N) F(fq_result, P)
    F(fq_result, status) F(fq_result, energy) F(fq_result, grad_gamma) F(fq_result, grad_beta)
    F(fq_result, t_submit) F(fq_result, t_start) F(fq_result, t_done)
    F(fq_server_counters, pending) F(fq_server_counters, kernel_launches)
    F(fq_server_counters, batched_requests) F(fq_server_counters, lane_requests)
    F(fq_server_counters, resident_sessions) F(fq_server_counters, resident_bytes)
    printf("FQ_SERVE_MAX_LAYERS %d\n", FQ_SERVE_MAX_LAYERS);
    return 0;
}
"""


def c_layout(tmp_path):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    src = tmp_path / "probe.c"
    src.write_text(PROBE)
    exe = tmp_path / "probe"
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    return dict((k, int(v)) for k, v in (line.split() for line in out.splitlines()))


def test_struct_layouts_match_header(fq, tmp_path):
    lay = c_layout(tmp_path)
    assert lay["FQ_SERVE_MAX_LAYERS"] == fq.SERVE_MAX_LAYERS
    for cname, pyt in (("fq_request", fq._Request), ("fq_result", fq._Result),
                       ("fq_server_counters", fq._Counters)):
        assert lay[cname] == ctypes.sizeof(pyt), cname
        for field, _ in pyt._fields_:
            key = f"{cname}.{field}"
            if key in lay:
                assert lay[key] == getattr(pyt, field).offset, key


def test_server_create_fails_cleanly_without_device(fq):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    with pytest.raises(fq.FQError):
        fq.Server(0, 1e9, 2)
