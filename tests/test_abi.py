"""The C ABI without a GPU: the library loads, exports every function
include/frehd_b200.h declares, and rejects bad arguments before any device
work."""
import ctypes as C
import os
import re

import pytest

from frehdc_b200 import native

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include",
                      "frehd_b200.h")


def declared_functions() -> list[str]:
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    names = re.findall(r"\b(frehd_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_header_declares_the_entry_points():
    names = declared_functions()
    for n in ["frehd_domain_create", "frehd_domain_step", "frehd_domain_run",
              "frehd_cg_solve_noalloc", "frehd_build_tables", "frehd_last_error"]:
        assert n in names


def test_library_exports_every_declared_function():
    lib = native.lib()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert missing == []


def test_status_strings():
    lib = native.lib()
    for code in range(0, 9):
        assert lib.frehd_status_string(code)


def test_noalloc_rejects_oversize_without_device_work():
    with pytest.raises(native.FrehdError) as e:
        native.cg_solve_noalloc(1024, 512, 1, 1, 1, 1, 1, 1e-12, 10)
    assert e.value.status == 1
    assert "262144" in str(e.value)


def test_domain_create_rejects_unsupported_option():
    from frehdc_b200 import deck as D
    cfg = D.config_dict(D.make_deck(D.DeckSpec(nx=16, ny=12, steps=2)))
    cfg["useminA"] = 1
    with pytest.raises(native.FrehdError) as e:
        native.Domain(cfg)
    assert e.value.status == 2


def test_domain_create_rejects_too_many_scalars():
    from frehdc_b200 import deck as D
    cfg = D.config_dict(D.make_deck(D.DeckSpec(nx=16, ny=12, steps=2)))
    cfg["nscalar"] = 5
    with pytest.raises(native.FrehdError) as e:
        native.Domain(cfg)
    assert e.value.status == 1 and "nscalar" in str(e.value)


def test_config_mirror_matches_the_c_struct(tmp_path):
    """The ctypes mirror of frehd_config has the C compiler's size and offsets."""
    import shutil
    import subprocess
    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    fields = [n for n, _ in native.Config._fields_]
    src = "#include <stdio.h>\n#include <stddef.h>\n#include \"frehd_b200.h\"\nint main(void){\n"
    src += 'printf("%zu\\n", sizeof(frehd_config));\n'
    src += "".join(f'printf("%zu\\n", offsetof(frehd_config, {n}));\n' for n in fields)
    src += "return 0;}\n"
    c = tmp_path / "probe.c"
    c.write_text(src)
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-I", os.path.dirname(HEADER), str(c), "-o", str(exe)], check=True)
    out = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True,
                                          check=True).stdout.split()]
    assert out[0] == C.sizeof(native.Config)
    assert out[1:] == [getattr(native.Config, n).offset for n in fields]


def test_server_create_fails_loudly_without_a_device():
    if native.device_count() > 0:
        pytest.skip("a CUDA device is visible")
    with pytest.raises(native.FrehdError):
        native.Server(1 << 30, 65536.0)
