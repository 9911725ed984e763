"""CPU tests of the C-ABI library: it loads and exports every declared symbol."""
import os
import re

from jf_2026_05_19_b200 import native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "jfem_gpu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(jfg_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = native.load()
    syms = declared_symbols()
    assert len(syms) >= 15
    for s in syms:
        assert hasattr(L, s), s
    assert set(syms) == set(native.EXPORTS)


def test_version_string():
    assert "sm_100a" in native.version()


def test_desc_layout_matches_header(tmp_path):
    """ctypes descriptor has the C struct's size and field offsets (compiled probe)."""
    import ctypes
    import subprocess
    from jf_2026_05_19_b200.abi import JfgModelDesc
    fields = [f for f, _ in JfgModelDesc._fields_]
    src = tmp_path / "probe.c"
    body = "".join(f'printf("%zu\\n", offsetof(jfg_model_desc, {f}));' for f in fields)
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "jfem_gpu.h"\n'
                   'int main(void){printf("%zu\\n", sizeof(jfg_model_desc));' + body + 'return 0;}')
    exe = tmp_path / "probe"
    cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    vals = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert vals[0] == ctypes.sizeof(JfgModelDesc)
    for f, off in zip(fields, vals[1:]):
        assert getattr(JfgModelDesc, f).offset == off, f
