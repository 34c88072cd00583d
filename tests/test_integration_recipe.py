"""The Rust crate's build recipe shown in INTEGRATION.md links.

The image has no Rust toolchain, so the crate itself is not compiled.  What can
be checked is what its build.rs and extern block claim: the `.cu` files listed
in `build.rs` are the library's own sources (the set the package's build
compiles), every function the `extern "C"` block of `src/ffi.rs` declares is a
function of include/efvm.h, and a C program that calls every one of them links
against the objects of exactly those files with the static CUDA runtime,
leaving no undefined symbol.  No GPU is needed: the program is linked and run,
but its calls sit behind a branch that is never taken.
"""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DOC = os.path.join(ROOT, "INTEGRATION.md")
HEADER = os.path.join(ROOT, "include", "efvm.h")


def recipe_files():
    doc = open(DOC).read()
    build_rs = doc[doc.index("fn main()"):]
    build_rs = build_rs[:build_rs.index("```")]
    return re.findall(r'\.file\(format!\("\{csrc\}/([a-z_0-9]+\.cu)"\)\)', build_rs)


def extern_block_functions():
    doc = open(DOC).read()
    block = doc[doc.index('extern "C" {'):]
    block = block[:block.index("\n}\n")]
    return re.findall(r"pub fn (efvm_[a-z_0-9]+)\(", block)


def header_functions():
    src = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    return set(re.findall(r"\b(efvm_[a-z_0-9]+)\s*\(", src))


def test_build_rs_lists_every_library_source():
    from dev_field_efvm_b200 import build
    files = recipe_files()
    assert len(files) == len(set(files))
    assert sorted(files) == sorted(build.SOURCES)


def test_extern_block_declares_only_header_functions():
    fns = extern_block_functions()
    assert len(fns) >= 30
    assert not set(fns) - header_functions(), sorted(set(fns) - header_functions())


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_c_program_calling_the_extern_block_links(tmp_path):
    from dev_field_efvm_b200 import build
    build.build()
    objs = [os.path.join(build.BUILD, f.replace(".cu", ".o")) for f in recipe_files()]
    for o in objs:
        assert os.path.exists(o), o
    fns = extern_block_functions()
    # every call takes zeroed arguments of the right types; the branch is never taken
    decls = open(HEADER).read()
    calls = []
    for f in fns:
        m = re.search(r"\b" + f + r"\s*\(([^;]*?)\)\s*;", re.sub(r"/\*.*?\*/", "", decls, flags=re.S), flags=re.S)
        assert m, f
        args = [a.strip() for a in m.group(1).split(",") if a.strip() and a.strip() != "void"]
        vals = []
        for a in args:
            if "*" in a or "[" in a:
                vals.append("0")
            elif a.startswith(("double", "float")):
                vals.append("0.0")
            else:
                vals.append("0")
        calls.append(f"        n += {f}({', '.join(vals)}) == 0;")
    prog = "\n".join([
        '#include <stdio.h>',
        '#include "efvm.h"',
        "int main(int argc, char** argv) {",
        "    int n = 0;",
        "    if (argc > 1000) {  /* never taken: the calls only have to link */",
        *calls,
        "    }",
        f'    printf("linked %d entry points\\n", {len(fns)});',
        "    return n;",
        "}",
    ])
    src = tmp_path / "calls.c"
    src.write_text(prog)
    obj = tmp_path / "calls.o"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), "-c", str(src),
                    "-o", str(obj)], check=True)
    exe = tmp_path / "calls"
    cuda_lib = os.path.join(os.path.dirname(os.path.dirname(build.nvcc())), "lib64")
    # the link step cc's CUDA build performs: the objects, the static CUDA runtime, libstdc++
    r = subprocess.run(["g++", str(obj), *objs, "-L", cuda_lib, "-lcudart_static", "-lrt", "-lpthread", "-ldl",
                        "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0 and f"linked {len(fns)} entry points" in out.stdout
