"""The C-ABI boundary without a GPU: the library loads, exports every
function include/bielcc_gpu.h declares, and the ctypes records have the
header's layout. No compute call is made here."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

from bielcc_b200 import abi, build
from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "bielcc_gpu.h")


def declared_functions():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int|void|const char\*)\s+(bielcc_\w+)\s*\(", txt, flags=re.M)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ("bielcc_ctx_create", "bielcc_mesh_create", "bielcc_field_EH", "bielcc_field_EH_device",
                 "bielcc_pair_op", "bielcc_integral_pnt", "bielcc_integral_seg_pnt", "bielcc_k0",
                 "bielcc_integral_1divr", "bielcc_assemble_K", "bielcc_integral", "bielcc_integral_seg"):
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = build.build()
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r" T (bielcc_\w+)", out))
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, missing
    L = C.CDLL(lib)  # loads without a device
    for n in declared_functions():
        assert hasattr(L, n)


def test_ctypes_layouts_match_header():
    src = r'''
    #include <stdio.h>
    #include <stddef.h>
    #include "bielcc_gpu.h"
    int main(void) {
      printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(bielcc_numparam),
             sizeof(bielcc_planewave),
             sizeof(bielcc_kernelparam), sizeof(bielcc_report), offsetof(bielcc_report, est_rel_l2),
             offsetof(bielcc_kernelparam, current), sizeof(bielcc_field_job), sizeof(bielcc_field_request),
             offsetof(bielcc_field_request, inc), sizeof(bielcc_assemble_request), sizeof(bielcc_server_stats),
             offsetof(bielcc_server_stats, p50_ms), sizeof(bielcc_batch_trace), offsetof(bielcc_batch_trace, admit_ms),
             sizeof(bielcc_stats));
      return 0; }
    '''
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        open(c, "w").write(src)
        exe = os.path.join(d, "t")
        subprocess.run(["gcc", "-I", os.path.dirname(HEADER), c, "-o", exe], check=True)
        sizes = list(map(int, subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()))
    assert sizes == [C.sizeof(abi.NumParam), C.sizeof(abi.PlaneWave), C.sizeof(abi.KernelParam),
                     C.sizeof(abi.Report), abi.Report.est_rel_l2.offset, abi.KernelParam.current.offset,
                     C.sizeof(abi.FieldJob), C.sizeof(abi.FieldRequest), abi.FieldRequest.inc.offset,
                     C.sizeof(abi.AssembleRequest), C.sizeof(abi.ServerStats), abi.ServerStats.p50_ms.offset,
                     C.sizeof(abi.BatchTrace), abi.BatchTrace.admit_ms.offset, C.sizeof(abi.Stats)]


def test_no_device_fails_loudly():
    """Without a visible CUDA device the product raises; nothing falls back to the CPU."""
    from bielcc_b200 import gpu

    try:
        import torch

        has_gpu = torch.cuda.is_available()
    except Exception:  # pragma: no cover
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present")
    with pytest.raises(gpu.BielccError) as e:
        gpu.Context(0)
    assert e.value.code in (abi.ERR_CUDA, abi.ERR_ARG)


def test_checkers_export_the_same_calls():
    import oracle

    for which in ("port", "ref"):
        if not oracle.available(which) and which == "ref":
            continue
        L, prefix = oracle.lib(which)
        for n in ("field_EH", "pair_op", "integral_pnt", "integral_seg_pnt", "integral", "integral_seg", "k0",
                  "integral_1divr",
                  "integral_grad1divr_seg", "integral_surf_simplepot_h_hs", "integral_seg_gradsimplepot_h_hs"):
            assert hasattr(L, prefix + n)
