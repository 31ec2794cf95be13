"""Host-side checks of the C ABI that need no GPU: the library loads, exports
every function include/rmhd2d.h declares, validates configurations, reports
a missing device cleanly and writes snapshots in the reference's format."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    text = (ROOT / "include" / "rmhd2d.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(rmhd2d_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from resistivemhd_gpu_b200 import _lib

    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), f"{n} declared in include/rmhd2d.h but not exported"
    bound = {n for n, _, _ in _lib.SIGNATURES}
    assert set(names) <= bound, f"missing ctypes signatures: {set(names) - bound}"


def test_abi_version_and_status_strings():
    from resistivemhd_gpu_b200 import _lib

    lib = _lib.load()
    assert lib.rmhd2d_abi_version() == 3
    for code, text in _lib.STATUS.items():
        assert lib.rmhd2d_status_string(code).decode() == text


def test_config_struct_layout_matches_defaults():
    from resistivemhd_gpu_b200 import _lib

    lib = _lib.load()
    cfg = _lib.Config()
    lib.rmhd2d_config_default(ctypes.byref(cfg))
    assert cfg.gamma_mhd == pytest.approx(5.0 / 3.0)
    assert cfg.cfl == 0.4 and cfg.eps == 1e-20 and cfg.bc == 0 and cfg.precision == 0
    assert cfg.stream is None


@pytest.mark.parametrize("field,value", [("nx", 11), ("ny", 5), ("dx", 0.0), ("gamma_mhd", 1.0), ("eta", -1.0),
                                         ("bc", 7), ("precision", 9)])
def test_create_rejects_bad_config(field, value):
    from resistivemhd_gpu_b200 import _lib

    lib = _lib.load()
    cfg = _lib.Config()
    lib.rmhd2d_config_default(ctypes.byref(cfg))
    cfg.nx, cfg.ny = 20, 20
    setattr(cfg, field, value)
    h = ctypes.c_void_p()
    st = lib.rmhd2d_create(ctypes.byref(cfg), ctypes.byref(h))
    assert st == 1 and not h.value
    assert lib.rmhd2d_last_error(None)


def test_create_without_device_fails_cleanly():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from resistivemhd_gpu_b200 import Solver, _lib

    with pytest.raises(_lib.RMHDError) as e:
        Solver(20, 20, 0.1, 0.1)
    assert e.value.status == 3


def test_null_arguments_are_rejected():
    from resistivemhd_gpu_b200 import _lib

    lib = _lib.load()
    assert lib.rmhd2d_create(None, None) == 1
    assert lib.rmhd2d_step_rk2(None) == 1
    assert lib.rmhd2d_destroy(None) == 0
    assert lib.rmhd2d_write_snapshot(None, None, 1, 1) == 1


def test_snapshot_format_matches_reference_save(tmp_path):
    """rmhd2d_write_snapshot emits what the reference's save() emits
    (resistiveMHD_2D.cu:198-244): every cell k = 0..nx*ny-1 in order, 8
    little-endian doubles rho, rhoU, rhoV, rhoW, bX, bY, bZ, e."""
    from resistivemhd_gpu_b200 import read_snapshot, setups, write_snapshot

    s = setups.random_smooth_state(9, 7)
    p = tmp_path / "x_3.bin"
    write_snapshot(str(p), s.state)
    raw = p.read_bytes()
    assert len(raw) == s.nx * s.ny * 8 * 8
    expect = b"".join(np.asarray(s.state[i, j], dtype="<f8").tobytes() for i in range(s.nx) for j in range(s.ny))
    assert raw == expect
    assert np.array_equal(read_snapshot(str(p), s.nx, s.ny), s.state)


def test_snapshot_matches_reference_binary_output(tmp_path):
    """The reference binary's final-state file (the fixture generator's output
    channel) and write_snapshot agree byte for byte."""
    from conftest import GOLDEN_CASES, load_golden
    from resistivemhd_gpu_b200 import write_snapshot

    _, _, final, _, _ = load_golden(GOLDEN_CASES[0])
    p = tmp_path / "f.bin"
    write_snapshot(str(p), final)
    assert p.read_bytes() == np.ascontiguousarray(final, dtype="<f8").tobytes()
