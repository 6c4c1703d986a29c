"""The C-ABI library loads and exports every entry point include/crowdphot_b200.h declares;
the ctypes struct layouts match the C compiler's (no device calls)."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

from crowdphot_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "crowdphot_b200.h")


def declared():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"CPB_API\s+[\w\s\*]+?\b(cpb_\w+)\s*\(", src)))


def test_header_declares_prototyped_symbols():
    names = declared()
    assert names, "no CPB_API declarations found"
    assert set(names) == set(_abi.PROTOTYPES), (set(names) ^ set(_abi.PROTOTYPES))


@pytest.mark.parametrize("path", [_abi.LIB_PATH, _abi.CHECKED_LIB_PATH], ids=["production", "checked"])
def test_library_exports_every_declared_symbol(path):
    if not os.path.exists(path):
        pytest.fail(f"library not built: {path}")
    lib = C.CDLL(path)
    for name in declared():
        assert hasattr(lib, name), name
    lib.cpb_version.restype = C.c_char_p
    assert b"sm_100a" in lib.cpb_version()


def test_struct_layouts_match_c():
    probe = r"""
#include <stdio.h>
#include <stddef.h>
#include "crowdphot_b200.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(cpb_psf_desc), sizeof(cpb_sim_params),
         sizeof(cpb_sim_result), sizeof(cpb_lm_params), sizeof(cpb_lm_result), sizeof(cpb_group_result),
         sizeof(cpb_tune_info), sizeof(cpb_server_config), sizeof(cpb_request_info));
  printf("%zu %zu %zu %zu %zu %zu\n", offsetof(cpb_sim_params, precision), offsetof(cpb_sim_result, n_passes),
         offsetof(cpb_sim_result, device_seconds), offsetof(cpb_lm_params, min_diagonal),
         offsetof(cpb_group_result, n_lsqr_iters), offsetof(cpb_group_result, device_seconds));
  return 0;
}
"""
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "probe.c")
        exe = os.path.join(d, "probe")
        open(src, "w").write(probe)
        subprocess.run(["gcc", "-I", os.path.dirname(HEADER), src, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split("\n")
    sizes = [int(v) for v in out[0].split()]
    offs = [int(v) for v in out[1].split()]
    assert sizes == [C.sizeof(_abi.PsfDesc), C.sizeof(_abi.SimParams), C.sizeof(_abi.SimResult),
                     C.sizeof(_abi.LMParams), C.sizeof(_abi.LMResultC), C.sizeof(_abi.GroupResult),
                     C.sizeof(_abi.TuneInfo), C.sizeof(_abi.ServerConfig), C.sizeof(_abi.RequestInfo)]
    assert offs == [_abi.SimParams.precision.offset, _abi.SimResult.n_passes.offset,
                    _abi.SimResult.device_seconds.offset, _abi.LMParams.min_diagonal.offset,
                    _abi.GroupResult.n_lsqr_iters.offset, _abi.GroupResult.device_seconds.offset]


def test_context_without_gpu_fails_loudly():
    # on a machine without a CUDA device the product path must refuse, not fall back
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import crowdphot_b200 as cpb
    with pytest.raises(cpb.CudaError):
        cpb.Context(0)
