"""The bindings INTEGRATION.md tells a maintainer to add must match the C ABI:
its ctypes structures have the sizes and field offsets of include/kdtree.h
(compiled here with gcc), and every argtypes list it gives has the arity of
the prototype it binds."""
import ctypes
import os
import re
import shutil
import subprocess

import pytest

from conftest import REPO
from corruscant_b200 import _native

DOC = open(os.path.join(REPO, "INTEGRATION.md")).read()
HEADER = open(os.path.join(REPO, "include", "kdtree.h")).read()


def _python_blocks():
    return re.findall(r"```python\n(.*?)```", DOC, flags=re.S)


def _class_source(name):
    """The class statement `class <name>(Structure):` from the guide's code."""
    for block in _python_blocks():
        m = re.search(r"^class %s\(Structure\):.*?(?=^\S|\Z)" % name, block, flags=re.S | re.M)
        if m:
            return m.group(0)
    raise AssertionError(f"INTEGRATION.md has no ctypes class {name}")


def _doc_struct(name):
    ns = {k: getattr(ctypes, k) for k in ("Structure", "POINTER", "c_int", "c_double",
                                          "c_longlong", "c_uint")}
    ns.update(node=_native.Node, datum=_native.Datum)
    exec(_class_source(name), ns)
    return ns[name]


def _c_layout(tmp_path, ctype, fields):
    """sizeof and offsetof of a struct of include/kdtree.h, from gcc."""
    if not shutil.which("gcc"):
        pytest.skip("gcc not available")
    src = "#include <stddef.h>\n#include <stdio.h>\n#include \"kdtree.h\"\nint main(void){\n"
    src += 'printf("%%zu\\n", sizeof(%s));\n' % ctype
    for f in fields:
        src += 'printf("%%zu\\n", offsetof(%s, %s));\n' % (ctype, f)
    src += "return 0;}\n"
    (tmp_path / "layout.c").write_text(src)
    exe = str(tmp_path / "layout")
    subprocess.run(["gcc", "-I", os.path.join(REPO, "include"), str(tmp_path / "layout.c"), "-o",
                    exe], check=True)
    vals = [int(x) for x in subprocess.check_output([exe]).split()]
    return vals[0], vals[1:]


@pytest.mark.parametrize("pyname,ctype", [("kdtree", "kdtree_t"), ("count_stats", "kd_count_stats")])
def test_guide_structures_match_the_header(tmp_path, pyname, ctype):
    S = _doc_struct(pyname)
    names = [f[0] for f in S._fields_]
    size, offsets = _c_layout(tmp_path, ctype, names)
    assert ctypes.sizeof(S) == size, (pyname, ctypes.sizeof(S), size)
    assert [getattr(S, n).offset for n in names] == offsets, pyname


def _arity(fn):
    proto = re.sub(r"/\*.*?\*/", "", HEADER, flags=re.S)
    m = re.search(r"\b%s\s*\(([^)]*)\)\s*;" % fn, proto, flags=re.S)
    assert m, fn
    args = [a for a in m.group(1).split(",") if a.strip() and a.strip() != "void"]
    return len(args)


def test_guide_argtypes_have_the_prototypes_arity():
    found = re.findall(r"kdlib\.(\w+)\.argtypes = \[(.*?)\]\n", DOC, flags=re.S)
    assert len(found) >= 2
    for fn, body in found:
        n = len([a for a in re.split(r",\s*(?![^\(]*\))", body.replace("\n", " ")) if a.strip()])
        assert n == _arity(fn), (fn, n, _arity(fn))
