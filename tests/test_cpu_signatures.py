"""The drop-in surface keeps the reference's signatures: every parameter of
PySIFT.__init__ (pysift/core.py:1184-1188), PySIFT.detectAndCompute
(pysift/core.py:2021), GPUPyStitch.__init__ (pysift/core.py:2429-2445) and
GPUPyStitch.stitch (pysift/core.py:3972) exists here, in the same position,
with the same default.  The reference's signatures are read from its source
with `ast` (nothing of it is imported or run); the test is skipped unless
PYSIFT_REFERENCE names the reference checkout.  Extra parameters here are
keyword-only."""
import ast
import inspect
import os

import pytest

from conftest import reference_root

REF_CORE = os.path.join(reference_root() or "", "pysift", "core.py")


def _ref_signature(cls_name, fn_name):
    tree = ast.parse(open(REF_CORE).read())
    for node in ast.walk(tree):
        if isinstance(node, ast.ClassDef) and node.name == cls_name:
            for f in node.body:
                if isinstance(f, ast.FunctionDef) and f.name == fn_name:
                    a = f.args
                    names = [x.arg for x in a.args][1:]
                    defaults = [None] * (len(a.args) - len(a.defaults)) + [ast.literal_eval(d) for d in a.defaults]
                    return list(zip(names, defaults[1:])), a.vararg is not None
    raise LookupError(f"{cls_name}.{fn_name}")


@pytest.mark.skipif(not os.path.isfile(REF_CORE), reason="PYSIFT_REFERENCE unset or not a reference checkout")
@pytest.mark.parametrize("cls_name,fn_name", [("PySIFT", "__init__"), ("PySIFT", "detectAndCompute"),
                                              ("GPUPyStitch", "__init__"), ("GPUPyStitch", "stitch")])
def test_signature_matches_reference(cls_name, fn_name):
    import pysift_b200
    ref, ref_varargs = _ref_signature(cls_name, fn_name)
    ours = inspect.signature(getattr(getattr(pysift_b200, cls_name), fn_name))
    params = [p for p in ours.parameters.values() if p.name != "self"]
    positional = [p for p in params if p.kind in (p.POSITIONAL_ONLY, p.POSITIONAL_OR_KEYWORD)]
    assert [p.name for p in positional] == [n for n, _ in ref]
    for p, (name, default) in zip(positional, ref):
        want = inspect.Parameter.empty if default is None and p.default is inspect.Parameter.empty else default
        assert p.default == want, f"{name}: default {p.default!r}, reference {default!r}"
    assert any(p.kind == p.VAR_POSITIONAL for p in params) == ref_varargs
    extra = [p for p in params if p.kind == p.KEYWORD_ONLY]
    assert all(p.default is not inspect.Parameter.empty for p in extra)
