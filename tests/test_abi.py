"""The C-ABI library loads on a CPU-only host and exports every entry point
that include/elemgpu.h declares.  No compute calls are made here."""
import ctypes
import subprocess

import elemental_b200 as eg


def test_library_loads_and_exports_every_declared_symbol():
    L = eg.lib()
    names = eg.exported_symbols()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", eg.LIB_PATH], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    assert set(names) <= exported
    # nothing else leaks out of the library (hidden visibility)
    assert {n for n in exported if n.startswith("egpu")} == set(names)


def test_error_strings_and_arguments_without_gpu():
    L = eg.lib()
    assert L.egpu_error_string(eg.NOT_HPD) == b"A was not numerically HPD"
    assert L.egpu_error_string(eg.SINGULAR) == b"Matrix was singular"
    assert L.egpu_create(None, 0) == -1  # EGPU_ERR_ARG
    h = ctypes.c_void_p()
    rc = L.egpu_create(ctypes.byref(h), 0)
    import torch
    if not torch.cuda.is_available():
        assert rc == -7  # EGPU_ERR_NO_DEVICE: fails loudly, no CPU fallback
    else:
        assert rc == 0
        L.egpu_destroy(h)


def test_enums_match_reference_values():
    # core/types_decl.hpp:104-155
    assert (eg.LOWER, eg.UPPER) == (0, 1)
    assert (eg.NORMAL, eg.TRANSPOSE, eg.ADJOINT) == (0, 1, 2)
    assert (eg.LEFT, eg.RIGHT) == (0, 1)
    assert (eg.NON_UNIT, eg.UNIT) == (0, 1)


def test_library_has_no_unresolved_own_symbols():
    out = subprocess.run(["nm", "-D", eg.LIB_PATH], capture_output=True, text=True).stdout
    undefined = [l.split()[-1] for l in out.splitlines() if " U " in l and "egpu" in l]
    assert not undefined, undefined


def test_header_is_plain_c(tmp_path):
    # bindings from C (cgo, JNI, ctypes users) include the header as C99
    import os
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = tmp_path / "uses_header.c"
    calls = "\n".join(f"  (void)&{n};" for n in eg.exported_symbols())
    src.write_text('#include "elemgpu.h"\nint main(void) {\n' + calls + "\n  return 0;\n}\n")
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I",
                    os.path.join(root, "include"), "-c", str(src), "-o", str(tmp_path / "uses_header.o")],
                   check=True, capture_output=True)


def test_device_vector_arguments_are_checked_before_any_call():
    import pytest
    import torch
    from elemental_b200 import _device_vec
    with pytest.raises(TypeError):
        _device_vec(torch.zeros(8, dtype=torch.int32), 8, "int32", 0)  # host tensor
    with pytest.raises(TypeError):
        _device_vec([0] * 8, 8, "int32", 0)
    with pytest.raises(KeyError):
        _device_vec(torch.zeros(8, dtype=torch.int32), 8, "int64", 0)
