"""The C ABI as a C or C++ caller sees it: include/cgli_fu_flow.h compiles
on its own as strict C99 and as C++11, and a C program that takes the
address of every function the header declares links against
libcgli_fu_flow.so (so every declaration has an extern "C" definition of
the same name).  No GPU is needed: nothing is called."""
import os
import re
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
HEADER = os.path.join(REPO, "include", "cgli_fu_flow.h")
LIB_DIR = os.path.join(REPO, "cgli_fu_flow_b200")


def _declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    text = re.sub(r"//[^\n]*", " ", text)
    names = re.findall(r"\b(cgli_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc not present")
@pytest.mark.parametrize("lang,std", [("c", "-std=c99"), ("c++", "-std=c++11")])
def test_header_compiles_alone(lang, std):
    cc = "gcc" if lang == "c" else "g++"
    r = subprocess.run([cc, std, "-Wall", "-Wextra", "-pedantic", "-Werror", "-fsyntax-only", "-x", lang, HEADER],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc not present")
def test_every_declared_function_links(tmp_path, cuda_lib):
    names = _declared_functions()
    assert len(names) > 50
    src = tmp_path / "abi.c"
    body = "\n".join(f"  (void *)&{n}," for n in names)
    src.write_text('#include <stdio.h>\n#include "cgli_fu_flow.h"\n'
                   f"static void *const fns[] = {{\n{body}\n}};\n"
                   "int main(void) { printf(\"%d\\n\", (int)(sizeof fns / sizeof fns[0])); return 0; }\n")
    exe = tmp_path / "abi"
    r = subprocess.run(["gcc", "-std=c99", "-I", os.path.dirname(HEADER), str(src), "-o", str(exe),
                        "-L", LIB_DIR, "-lcgli_fu_flow", f"-Wl,-rpath,{LIB_DIR}"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    # the program loads the library (every symbol resolves) and runs on a
    # machine without a GPU: it only prints the table's size
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert int(r.stdout) == len(names)
