"""The C-ABI library loads and exports every symbol include/cmh_fof.h
declares; without a usable GPU the compute entry points return an error
status instead of crashing or falling back to the CPU."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from cm_halofinder_b200 import _abi

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                      "include", "cmh_fof.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(cmh_[a-z_0-9]+)\s*\(", src)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for required in ("cmh_fof_run", "cmh_plan_create", "cmh_plan_run", "cmh_catalog_free",
                     "cmh_read_parameterfile", "cmh_write_halos", "cmh_write_info",
                     "cmh_fof_run_batch", "cmh_last_error"):
        assert required in names


def test_library_exports_every_declared_symbol(native_lib):
    for name in declared_functions():
        assert hasattr(native_lib, name), name
    assert set(declared_functions()) == set(_abi.SIGNATURES)
    assert native_lib.cmh_abi_version() == 2


def test_structs_match_header_layout(tmp_path):
    """sizeof of every ABI struct, computed by the C compiler from the
    header, equals the ctypes mirror's."""
    import subprocess
    structs = {"cmh_fof_params": _abi.FofParams, "cmh_particles": _abi.Particles,
               "cmh_stats": _abi.Stats, "cmh_catalog": _abi.Catalog,
               "cmh_run_parameters": _abi.RunParameters, "cmh_limits": _abi.Limits}
    prog = tmp_path / "sz.c"
    prog.write_text('#include <stdio.h>\n#include "cmh_fof.h"\nint main(void){\n' + "".join(
        f'printf("%zu\\n", sizeof({k}));\n' for k in structs) + "return 0;}\n")
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I", os.path.dirname(HEADER), str(prog), "-o", str(exe)], check=True)
    sizes = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True,
                                            check=True).stdout.split()]
    for (name, ct), sz in zip(structs.items(), sizes):
        assert C.sizeof(ct) == sz, name


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device error path")
def test_compute_without_device_fails_loudly(native_lib):
    from cm_halofinder_b200 import CmhError, FofConfig, fof
    pos = np.zeros((4, 3), np.float32)
    cfg = FofConfig(lo=(0, 0, 0), hi=(1, 1, 1), boundary=0.1, linklength=0.2)
    with pytest.raises(CmhError) as e:
        fof(pos, pos.copy(), cfg)
    assert e.value.status in (3, 9)
    h = C.c_void_p()
    p = cfg.to_c()
    st = native_lib.cmh_plan_create(C.byref(h), C.byref(p), 4, 0, 0)
    assert st in (3, 9) and not h.value


def test_invalid_arguments_are_reported(native_lib):
    cat = _abi.Catalog()
    assert native_lib.cmh_fof_run(None, None, C.byref(cat), 0, None) == 1
    buf = C.create_string_buffer(256)
    assert native_lib.cmh_last_error(buf, 256) > 0
    native_lib.cmh_catalog_free(C.byref(cat))   # freeing an empty catalog is harmless
    native_lib.cmh_catalog_free(None)
