"""The C ABI (include/yuzen_b200.h): the library is built for sm_100a, loads,
and exports every entry point the header declares.  No compute call here:
this runs without a GPU."""
import re
import subprocess
from pathlib import Path

import yuzen_b200

HEADER = Path(__file__).resolve().parents[1] / "include" / "yuzen_b200.h"


def declared_symbols():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(yz_[a-z0-9_]+)\s*\(", text)))


def test_header_and_binding_agree():
    assert declared_symbols() == sorted(yuzen_b200.EXPORTED_SYMBOLS)


def test_library_loads_and_exports_every_symbol():
    L = yuzen_b200.lib()
    for name in declared_symbols():
        assert hasattr(L, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", str(yuzen_b200.lib_path())],
                         capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r" T (yz_[a-z0-9_]+)", out))
    assert set(declared_symbols()) <= exported


def test_library_is_built_for_sm100a_only():
    from yuzen_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
    assert "-fmad=false" in build._flags(Path("x.cu"))


def test_last_error_is_callable_without_gpu():
    assert isinstance(yuzen_b200.lib().yz_last_error(), bytes)
