"""The C-ABI library: it loads, exports every entry point include/nimbus_cuda.h
declares, its argument blocks have the layout the ctypes binding assumes, and
it refuses to run without an sm_100 device (there is no CPU fallback).  No
compute call is made here."""
import ctypes
import re
import subprocess
from pathlib import Path

import pytest

from nimbus_b200 import cuda

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "nimbus_cuda.h"


def declared_functions():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:nimbus_status|void\*?|const char\*|int|uint64_t)\s+(nimbus_cuda_\w+)\(",
                                 text, re.M)))


def test_header_declares_what_binding_expects():
    assert set(declared_functions()) == set(cuda.EXPORTED_SYMBOLS)


def test_library_exports_every_declared_symbol():
    lib = cuda.load_library()
    for name in declared_functions():
        assert hasattr(lib, name), name
    assert lib.nimbus_cuda_abi_version() == 1


def _c_layout(struct_name, fields, tmp_path):
    src = tmp_path / "layout.c"
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void){",
             f'printf("%zu\\n", sizeof({struct_name}));']
    lines += [f'printf("%zu\\n", offsetof({struct_name}, {f}));' for f in fields]
    lines.append("return 0;}")
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", str(src), "-o", str(exe)], check=True)
    vals = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    return vals[0], vals[1:]


@pytest.mark.parametrize("struct_name,cls", [
    ("nimbus_acoustic_fused_args", cuda.AcousticFusedArgs),
    ("nimbus_acoustic_batched_args", cuda.AcousticBatchedArgs),
    ("nimbus_scalar_transport_args", cuda.ScalarTransportArgs),
])
def test_argument_block_layout_matches_header(struct_name, cls, tmp_path):
    fields = [f for f, _ in cls._fields_]
    size, offsets = _c_layout(struct_name, fields, tmp_path)
    assert size == ctypes.sizeof(cls)
    assert offsets == [getattr(cls, f).offset for f in fields]


def test_no_device_is_an_error_not_a_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(cuda.NimbusCudaError) as exc:
        cuda.Context(0)
    assert exc.value.status == 6  # NIMBUS_ERR_NO_DEVICE
    backend = cuda.CudaComputeBackend()
    assert backend.initialize() is False and "NO_DEVICE" in backend.last_error
