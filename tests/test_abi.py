"""The C ABI without a GPU: every symbol of include/btd.h is exported, the ctypes mirrors match the
C layout, and the solver refuses to run without a CUDA device (there is no CPU fallback)."""
import ctypes as C
import os
import re
import subprocess

import pytest

import btd_b200 as btd
from btd_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "btd.h")


def declared():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^int (btd_\w+)\(", text, re.M)))


def test_every_declared_symbol_is_exported_and_bound():
    lib = C.CDLL(_abi.LIB_PATH)
    names = declared()
    assert len(names) >= 40
    for n in names:
        assert hasattr(lib, n), n
        assert n in _abi.SIGNATURES, n


def test_struct_layouts_match_the_c_compiler(tmp_path):
    src = tmp_path / "sz.c"
    structs = ["btd_yarn", "btd_material", "btd_wear", "btd_layer_spec", "btd_layer_info", "btd_scene", "btd_params"]
    body = "".join(f'printf("%zu\\n", sizeof({s}));' for s in structs)
    src.write_text(f'#include <stdio.h>\n#include "btd.h"\nint main(void){{{body}return 0;}}\n')
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    sizes = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    mirrors = [_abi.Yarn, _abi.Material, _abi.Wear, _abi.LayerSpec, _abi.LayerInfo, _abi.SceneC, _abi.Params]
    assert sizes == [C.sizeof(m) for m in mirrors]


def test_default_params_are_the_reference_gpu_defaults():
    p = btd.default_params()
    assert abs(p.h - 1 / 120) < 1e-15 and p.newton_iterations == 2 and p.pcg_iterations == 2
    assert p.coarse_sweeps == 2 and p.max_coarsest_nodes == 400 and p.line_search == 1 and p.lag_coarse == 1
    assert p.newton_max == 2 and abs(p.newton_tolerance - 1e-5) < 1e-12 and p.self_contact == 1
    assert p.overlap_launches == 1  # extension: launch overlap only, same results


def _has_device():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_device(), reason="a CUDA device is present")
def test_create_fails_loudly_without_a_device():
    sc = btd.configs.hanging_patch(8, 0.1)
    with pytest.raises(_abi.BtdError) as e:
        btd.GpuSolver(sc)
    assert e.value.rc == -3
    assert "no CUDA device" in str(e.value)
