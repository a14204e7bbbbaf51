"""The C-ABI library loads without a GPU and exports every symbol of include/mgglam.h."""
import ctypes
import os
import re

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "mgglam.h")
LIB = os.path.join(ROOT, "mg-glam-durham_b200", "libmgglam_b200.so")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|int64_t|const char\*)\s+(mgg_\w+)\s*\(", text, re.M)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ("mgg_create", "mgg_density", "mgg_scalar_field", "mgg_potential", "mgg_potential_mg",
              "mgg_move", "mgg_power", "mgg_destroy"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    assert os.path.exists(LIB), "build with `make -C mg-glam-durham_b200`"
    lib = ctypes.CDLL(LIB)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_python_mirror_lists_all_symbols():
    import mgglam_b200
    assert sorted(mgglam_b200.EXPORTED_SYMBOLS) == declared_symbols()


def test_create_without_device_fails_cleanly():
    """No CUDA device here: mgg_create must return an error code, not crash."""
    from conftest import gpu_available
    import mgglam_b200 as m
    if gpu_available():
        return
    try:
        m.Box(m.make_config(16, 8, 16.0))
    except m.MGGError as e:
        assert e.code in (2, 7)
    else:
        raise AssertionError("mgg_create succeeded without a GPU")


def test_create_rejects_unknown_precision():
    """The precision form is checked before any device call: an unknown value is
    MGG_ERR_ARG with or without a GPU."""
    import mgglam_b200 as m
    try:
        m.Box(m.make_config(16, 8, 16.0, precision=2))
    except m.MGGError as e:
        assert m.ERR_NAMES[e.code] == "ARG", e
    else:
        raise AssertionError("mgg_create accepted precision 2")


def _c_layout(struct, fields, tmp_path):
    """sizeof and offsetof of a header struct, compiled with the host C compiler."""
    import subprocess
    src = tmp_path / "layout.c"
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void){",
             f'printf("%zu\\n", sizeof({struct}));']
    lines += [f'printf("%zu\\n", offsetof({struct}, {f}));' for f in fields]
    lines.append("return 0;}")
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    return [int(v) for v in out]


def test_struct_layouts_match_header(tmp_path):
    import mgglam_b200 as m
    for struct, cls in (("mgg_config", m.MggConfig), ("mgg_mg_report", m.MggReport),
                        ("mgg_ic_params", m.MggIcParams), ("mgg_step_state", m.MggStepState),
                        ("mgg_request", m.MggRequest), ("mgg_result_info", m.MggResultInfo),
                        ("mgg_pm_header", m.MggPmHeader)):
        names = [f[0] for f in cls._fields_]
        got = _c_layout(struct, names, tmp_path)
        assert got[0] == ctypes.sizeof(cls), struct
        assert got[1:] == [getattr(cls, n).offset for n in names], struct


def test_forms_without_device_fail_cleanly():
    from conftest import gpu_available
    import mgglam_b200 as m
    lib = m.load_library()
    h = ctypes.c_void_p()
    if not gpu_available():
        assert lib.mgg_server_create(0, 1.0, 2, ctypes.byref(h)) == 7   # MGG_ERR_NO_DEVICE
    assert lib.mgg_step(None, None) == 1                             # MGG_ERR_ARG
    cfg = m.make_config(1024, 512, 1024.0)
    nbytes = lib.mgg_box_bytes(ctypes.byref(cfg))
    # 512^3 particles on a 1024^3 mesh: about 25 GB on the device
    assert 20e9 < nbytes < 30e9
