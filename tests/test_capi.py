"""The C ABI (include/yuzen_b200.h): the library is built for sm_100a, loads,
and exports every entry point the header declares.  No compute call here:
this runs without a GPU."""
import ctypes
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


def test_struct_layouts_match_the_header(tmp_path):
    """Every struct the C ABI passes (yz_settings, yz_step_params,
    yz_step_stats, yz_cz_params, yz_cz_stats, yz_learned_cfg) has the size and
    the field offsets of its ctypes mirror: a C program built against the
    header with the host's C compiler prints sizeof and offsetof."""
    from yuzen_b200 import cz, learned, step
    mirrors = {"yz_settings": yuzen_b200._Settings, "yz_step_params": step.StepParams,
               "yz_step_stats": step.StepStats, "yz_cz_params": cz.CzParams, "yz_cz_stats": cz.CzStats,
               "yz_learned_cfg": learned.LearnedConfig}
    lines = ['#include <stddef.h>', '#include <stdio.h>', f'#include "{HEADER}"', "int main(void) {"]
    for cname, py in mirrors.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-o", str(exe), str(src)], check=True, capture_output=True)
    got = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    want = []
    for cname, py in mirrors.items():
        want.append(f"{cname} size {ctypes.sizeof(py)}")
        want += [f"{cname} {fname} {getattr(py, fname).offset}" for fname, _ in py._fields_]
    assert [g for g in got if g] == want
