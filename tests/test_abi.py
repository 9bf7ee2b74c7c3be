"""The drop-in boundary: libfaf_b200.so loads, exports every function that
include/*.h declares, and the public structs keep the reference's field
offsets (golden abi.json, compiled from the reference header).  CPU only:
no compute call needs a GPU here."""
import json
import os
import re
import subprocess
import sys
import tempfile

import pytest

from conftest import ROOT

INCLUDE = os.path.join(ROOT, "include")
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))


def declared_functions():
    names = set()
    for h in os.listdir(INCLUDE):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(INCLUDE, h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        # drop the extern "C" guards and other preprocessor lines
        text = re.sub(r"#ifdef __cplusplus.*?#endif", "", text, flags=re.S)
        text = "\n".join(l for l in text.splitlines() if not l.lstrip().startswith("#"))
        # drop inline bodies
        depth, out = 0, []
        for ch in text:
            if ch == "{":
                depth += 1
            elif ch == "}":
                depth -= 1
                continue
            if depth == 0:
                out.append(ch)
        text = "".join(out)
        for m in re.finditer(r"([A-Za-z_][A-Za-z0-9_\s\*]*?)\b([a-z_][a-z0-9_]*)\s*\(([^;{)]*)\)\s*;",
                             text):
            head, name = m.group(1), m.group(2)
            if "typedef" in head or "static" in head or "(*" in head:
                continue
            if name.startswith(("faf_", "chirp_")):
                names.add(name)
    return names


def exported_symbols(path):
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True,
                         check=True).stdout
    syms = set()
    for line in out.splitlines():
        parts = line.split()
        if len(parts) >= 3 and parts[1] in ("T", "W"):
            syms.add(parts[2].split("@")[0])
    return syms


def test_library_loads_and_exports_every_declared_symbol():
    import fastandfourier_b200 as F
    F.lib()  # loads (builds first if missing)
    decl = declared_functions()
    assert {"faf_execute", "faf_create_fft", "faf_create_rfft", "chirp_compile",
            "faf_execute_batched", "faf_cuda_set_stream"} <= decl
    exported = exported_symbols(F.C.LIB_PATH)
    missing = sorted(decl - exported)
    assert not missing, f"declared but not exported: {missing}"


ABI_PROGRAM_SRC = None


def compile_offsets(include_dir):
    import gen_golden
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "abi.c")
        exe = os.path.join(d, "abi")
        prog = gen_golden.ABI_PROGRAM.replace(
            'printf("}\\n");',
            'printf(",\\"faf_transform.device_plan\\": %zu, \\"sizeof.faf_transform\\": %zu\\n}\\n",'
            ' offsetof(faf_transform, device_plan), sizeof(faf_transform));')
        with open(src, "w") as f:
            f.write(prog)
        subprocess.run(["gcc", "-std=c11", "-I", include_dir, src, "-o", exe], check=True)
        return json.loads(subprocess.run([exe], capture_output=True, text=True,
                                         check=True).stdout)


def test_struct_layout_matches_reference_header():
    with open(os.path.join(ROOT, "tests", "golden", "abi.json")) as f:
        ref = json.load(f)
    ours = compile_offsets(INCLUDE)
    for k, v in ref.items():
        assert ours[k] == v, f"{k}: ours {ours[k]} reference {v}"
    # one appended trailing field, nothing moved
    last = max(v for k, v in ref.items() if k.startswith("faf_transform."))
    assert ours["faf_transform.device_plan"] > last
    assert ours["sizeof.faf_transform"] == ours["faf_transform.device_plan"] + 8


def test_ctypes_mirror_matches_header():
    import ctypes
    import fastandfourier_b200 as F
    ours = compile_offsets(INCLUDE)
    assert ctypes.sizeof(F.C.faf_transform) == ours["sizeof.faf_transform"]
    assert ctypes.sizeof(F.C.faf_config) == ours["sizeof.faf_config"]
    assert F.C.faf_transform.device_plan.offset == ours["faf_transform.device_plan"]
    assert F.C.faf_transform.cfg.offset == ours["faf_transform.cfg"]
    assert F.C.faf_transform.user_aux_n.offset == ours["faf_transform.user_aux_n"]


def test_header_compiles_as_cxx_and_c():
    with tempfile.TemporaryDirectory() as d:
        for lang, comp in (("c", "gcc"), ("cpp", "g++")):
            src = os.path.join(d, f"t.{lang}")
            with open(src, "w") as f:
                f.write('#include "fastandfourier.h"\n#include "chirp.h"\n#include "faf_cuda.h"\n'
                        "int main(void){ faf_config c = faf_config_init(8); "
                        "faf_buffer b = faf_buffer_split(0,0,8); (void)b; "
                        "return (int)faf_config_inverse(c).dir - 1; }\n")
            subprocess.run([comp, "-Wall", "-Werror", "-I", INCLUDE, "-c", src, "-o",
                            os.path.join(d, f"t_{lang}.o")], check=True)


def test_backend_enum_is_additive():
    ours = compile_offsets(INCLUDE)
    assert ours["enum.FAF_BACKEND_JIT"] == 2
    import fastandfourier_b200 as F
    assert F.B_CUDA == 3
