"""The C-ABI library loads on a machine without a GPU, exports every entry
point include/egtb_gpu.h declares, and reports errors instead of falling back
to the CPU."""
import ctypes
import os
import re

import numpy as np

import helpers as H

HEADER = os.path.join(H.ROOT, "include", "egtb_gpu.h")


def declared_symbols() -> list[str]:
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^EGTB_API\s+[\w\s\*]+?\b(egtb_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_the_binding_set():
    names = declared_symbols()
    assert len(names) >= 20
    assert sorted(H.pkg()._native.exported_symbols()) == names


def test_library_exports_every_declared_symbol():
    N = H.pkg()._native
    lib = N.lib()
    for name in declared_symbols():
        assert getattr(lib, name, None) is not None, name


def test_library_is_in_tree_and_built_for_sm100a():
    N = H.pkg()._native
    assert N.LIB_PATH.startswith(os.path.join(H.ROOT, "2048endgametablebase_b200"))
    assert b"sm_100a" in N.lib().egtb_version()


def test_struct_layouts_match_header(tmp_path):
    """ctypes mirrors of the ABI structs have the C compiler's sizes and offsets."""
    import subprocess
    N = H.pkg()._native
    fields = {
        "egtb_pattern_spec": N.PatternSpecC,
        "egtb_run_options": N.RunOptionsC,
        "egtb_build_stats": N.BuildStatsC,
        "egtb_kernel_time": N.KernelTimeC,
        "egtb_batch_params": N.BatchParamsC,
        "egtb_batch_stats": N.BatchStatsC,
    }
    lines = ["#include <stdio.h>", "#include <stddef.h>", f'#include "{HEADER}"', "int main(void) {"]
    for cname, cls in fields.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0; }")
    src = tmp_path / "abi.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "abi"
    subprocess.run(["gcc", "-o", str(exe), str(src)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = dict(line.rsplit(" ", 1) for line in out if line)
    for cname, cls in fields.items():
        assert int(got[f"{cname} size"]) == ctypes.sizeof(cls), cname
        for fname, _ in cls._fields_:
            assert int(got[f"{cname}.{fname}"]) == getattr(cls, fname).offset, (cname, fname)


def test_no_device_is_an_error_not_a_fallback():
    N = H.pkg()._native
    if N.device_count() > 0:
        return  # only meaningful on a machine without a GPU
    case = H.cases()["44_64_float32"]
    spec, o = H.spec_options(case, "/tmp/egtb_nodev_")
    F = H.fc()
    try:
        F.run_pattern_build(H.seeds(case), spec, o)
    except RuntimeError as e:
        assert "EGTB_ERR" in str(e)
    else:
        raise AssertionError("a build without a device must fail")
    b = np.zeros(1, dtype=np.uint64)
    out = np.zeros(4, dtype=np.uint64)
    assert N.lib().egtb_move_all_dir(0, b.ctypes.data, 1, out.ctypes.data) != 0


def test_error_message_buffer():
    N = H.pkg()._native
    buf = ctypes.create_string_buffer(8)
    assert N.lib().egtb_last_error(buf, 8) == 0
    assert N.lib().egtb_last_error(None, 0) == -1
