"""The C-ABI library loads and exports every symbol include/filianore_gpu.h declares
(no compute calls: runs without a GPU)."""
import ctypes
import os
import re

import filianore_b200 as fb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            text = open(os.path.join(ROOT, "include", h)).read()
            names |= set(re.findall(r"FL_API\s+[\w\s\*]+?\b(fl_\w+)\s*\(", text))
    return names


def test_header_declares_the_entry_points():
    names = declared_symbols()
    assert {"fl_context_create", "fl_scene_create", "fl_trace_closest", "fl_trace_occluded", "fl_render"} <= names


def test_library_exports_every_declared_symbol():
    lib = fb.lib()
    for name in declared_symbols():
        assert hasattr(lib, name), name
    assert set(fb.EXPORTED) >= declared_symbols() - set()


def test_status_strings_and_no_device_error():
    lib = fb.lib()
    assert lib.fl_status_string(0) == b"FL_OK"
    assert lib.fl_status_string(-5) == b"FL_ERR_TRAVERSAL"
    # null tables are rejected before any device work
    h = ctypes.c_void_p()
    assert lib.fl_context_create(0, None, ctypes.byref(h)) == fb.FL_ERR_INVALID


def test_ctypes_structs_match_the_header(tmp_path):
    """Every ctypes mirror in filianore_b200.types has the C struct's size and field offsets:
    a C program built against include/filianore_gpu.h prints them (gcc, no GPU)."""
    import subprocess

    from filianore_b200 import types as T
    structs = [(name, cls) for name, cls in vars(T).items()
               if isinstance(cls, type) and issubclass(cls, ctypes.Structure) and name.startswith("fl_")]
    assert len(structs) >= 10
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "filianore_gpu.h"', "int main(void) {"]
    for name, cls in structs:
        lines.append(f'    printf("{name} %zu\\n", sizeof({name}));')
        for field, _ in cls._fields_:
            lines.append(f'    printf("{name}.{field} %zu\\n", offsetof({name}, {field}));')
    lines += ["    return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(src)], check=True)
    got = dict(line.rsplit(" ", 1) for line in subprocess.run([str(exe)], check=True, capture_output=True,
                                                                text=True).stdout.splitlines())
    for name, cls in structs:
        assert int(got[name]) == ctypes.sizeof(cls), name
        for field, _ in cls._fields_:
            assert int(got[f"{name}.{field}"]) == getattr(cls, field).offset, (name, field)


def test_constants_match_the_header():
    """Every #define and enum constant of include/filianore_gpu.h has the same value in the
    ctypes binding (filianore_b200.types), where the binding names it."""
    from filianore_b200 import types as T
    text = open(os.path.join(ROOT, "include", "filianore_gpu.h")).read()
    consts = {m.group(1): int(m.group(2)) for m in re.finditer(r"#define\s+(FL_\w+)\s+(-?\d+)\b", text)}
    for body in re.findall(r"enum\s*\{([^}]*)\}", text):
        body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
        for m in re.finditer(r"(FL_\w+)\s*=\s*(-?\d+)", body):
            consts[m.group(1)] = int(m.group(2))
    assert "FL_GUIDE_PARAMS" in consts and "FL_RENDER_LOBE_DEPTHS" in consts
    checked = 0
    for name, value in consts.items():
        if hasattr(T, name):
            assert getattr(T, name) == value, name
            checked += 1
    assert checked >= 20
