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
    return sorted(set(re.findall(r"^\s*(?:nimbus_status|void\*?|const char\*|int|uint64_t|size_t)\s+(nimbus_\w+)\(",
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
    ("nimbus_slow_args", cuda.SlowArgs),
    ("nimbus_kessler_args", cuda.KesslerArgs),
    ("nimbus_eos_args", cuda.EosArgs),
    ("nimbus_sound_speed_args", cuda.SoundSpeedArgs),
    ("nimbus_slow_apply_args", cuda.SlowApplyArgs),
    ("nimbus_kessler_pointwise_args", cuda.KesslerPointwiseArgs),
    ("nimbus_kessler_sedimentation_args", cuda.KesslerSedimentationArgs),
    ("nimbus_cgrid_slow_tendencies_args", cuda.CgridSlowTendenciesArgs),
    ("nimbus_device_info", cuda.DeviceInfo),
    ("nimbus_boundary_args", cuda.BoundaryArgs),
    ("nimbus_state_relaxation_args", cuda.StateRelaxationArgs),
    ("nimbus_cell_centre_args", cuda.CellCentreArgs),
    ("nimbus_smagorinsky_args", cuda.SmagorinskyArgs),
    ("nimbus_sgs_apply_args", cuda.SgsApplyArgs),
    ("nimbus_sgs_stability", cuda.SgsStability),
    ("nimbus_sgs_step_args", cuda.SgsStepArgs),
    ("nimbus_history_args", cuda.HistoryArgs),
    ("nimbus_member_desc", cuda.MemberDesc),
    ("nimbus_engine_tuning", cuda.EngineTuning),
    ("nimbus_member_state", cuda.MemberState),
])
def test_argument_block_layout_matches_header(struct_name, cls, tmp_path):
    fields = [f for f, _ in cls._fields_]
    size, offsets = _c_layout(struct_name, fields, tmp_path)
    assert size == ctypes.sizeof(cls)
    assert offsets == [getattr(cls, f).offset for f in fields]


def test_reference_backend_adapter_exports():
    """The ComputeBackend adapter loads and exposes its factory hooks (no
    backend is created here)."""
    path = ROOT / "nimbus_b200" / "lib" / "libnimbus_reference_backend.so"
    if not path.exists():
        pytest.skip("adapter not built (no reference headers)")
    lib = ctypes.CDLL(str(path))
    assert hasattr(lib, "nimbus_cuda_create_compute_backend")
    assert hasattr(lib, "nimbus_cuda_destroy_compute_backend")


def test_no_device_is_an_error_not_a_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(cuda.NimbusCudaError) as exc:
        cuda.Context(0)
    assert exc.value.status == 6  # NIMBUS_ERR_NO_DEVICE
    backend = cuda.CudaComputeBackend()
    assert backend.initialize() is False and "NO_DEVICE" in backend.last_error


def test_argument_blocks_keep_their_arrays_alive():
    """Argument blocks hold raw pointers; the binding must keep every array
    they point at alive even when the caller passed temporaries."""
    import gc

    import numpy as np

    shape = (6, 5, 4)

    def tmp():
        return np.random.default_rng(0).random(shape).astype(np.float32)

    a = cuda.transport_args([tmp(), tmp()], [tmp(), tmp()], [0, 1], tmp(), tmp(), tmp(), tmp(), tmp(), 1.0,
                            (1.0, 1.0, 1.0))
    st = {k: tmp() for k in ("u", "v", "w", "rho", "p", "theta")}
    b = cuda.batched_args(st, np.ones(4), np.ones(4), 0.1, 2, (1.0, 1.0, 1.0), (1, 1, 1, 1, 1, 0), tmp(), tmp(),
                          tmp(), 0.5, None, np.zeros(2 * 11 * 4, np.float32), tmp())
    del st
    gc.collect()

    def kept_addresses(block):
        out = set()
        for item in block._keep:
            items = item.values() if isinstance(item, dict) else (item if isinstance(item, list) else [item])
            for arr in items:
                if isinstance(arr, np.ndarray):
                    out.add(arr.ctypes.data)
        return out

    for block, names in ((a, ("rho_end", "rho_begin", "mass_flux_x", "mass_flux_y", "mass_flux_z")),
                         (b, ("u", "rho", "theta", "rho0_base", "mass_flux_z", "wave_history_output",
                              "density_begin"))):
        kept = kept_addresses(block)
        for name in names:
            addr = ctypes.cast(getattr(block, name), ctypes.c_void_p).value
            assert addr in kept, name
    for i in range(2):
        assert ctypes.cast(a.q_in[i], ctypes.c_void_p).value in kept_addresses(a)
