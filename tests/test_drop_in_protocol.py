"""The B200 backend offers everything the reference's callers use of a backend.

Read from the reference's source (no import, no GPU): the ``Backend`` base
class (src/backends/base.py:81-201) -- its abstract and inherited methods with
their parameters, the attributes its constructor sets -- and every attribute
the reference's callers read off a backend object in src/timestepping/march.py,
src/api.py, src/sweep.py, src/cli.py and src/sensitivity.py.  ``B200Backend``
must provide each, with the same positional parameters.  The GPU test
``test_gpu_drop_in.py`` replays the calls themselves.  Skipped where no
reference checkout is present (set NOZZLE_REFERENCE to one).
"""

from __future__ import annotations

import ast
import inspect
import os

import pytest

from conftest import pkg

REFERENCE = os.environ.get("NOZZLE_REFERENCE", "/root/reference")
pytestmark = pytest.mark.skipif(not os.path.exists(os.path.join(REFERENCE, "src", "backends", "base.py")),
                                reason="no reference checkout")
CALLERS = ("src/timestepping/march.py", "src/api.py", "src/sweep.py", "src/cli.py", "src/sensitivity.py")
BACKEND_NAMES = {"backend", "bk"}


def _tree(rel):
    with open(os.path.join(REFERENCE, rel)) as fh:
        return ast.parse(fh.read())


def _backend_class():
    for node in ast.walk(_tree("src/backends/base.py")):
        if isinstance(node, ast.ClassDef) and node.name == "Backend":
            return node
    raise AssertionError("class Backend not found")


def _reference_methods():
    out = {}
    for node in _backend_class().body:
        if isinstance(node, ast.FunctionDef) and not node.name.startswith("_"):
            abstract = any(isinstance(d, ast.Name) and d.id == "abstractmethod" for d in node.decorator_list)
            out[node.name] = ([a.arg for a in node.args.args[1:]], abstract)
    return out


def _init_attributes(cls_node):
    names = set()
    for node in cls_node.body:
        if isinstance(node, ast.FunctionDef) and node.name == "__init__":
            for sub in ast.walk(node):
                if isinstance(sub, ast.Attribute) and isinstance(sub.value, ast.Name) and sub.value.id == "self" \
                        and isinstance(sub.ctx, ast.Store):
                    names.add(sub.attr)
        elif isinstance(node, (ast.Assign, ast.AnnAssign)):
            targets = node.targets if isinstance(node, ast.Assign) else [node.target]
            names.update(t.id for t in targets if isinstance(t, ast.Name))
    return names


def _our_attributes():
    B = pkg("backend").B200Backend
    src = inspect.getsource(B)
    import textwrap

    cls = ast.parse(textwrap.dedent(src)).body[0]
    return _init_attributes(cls) | {n for n in dir(B) if not n.startswith("__")}


def test_every_backend_method_is_provided_with_its_parameters():
    B = pkg("backend").B200Backend
    methods = _reference_methods()
    assert {"residual", "inverse_mass", "limit", "time_step", "norm"} <= {m for m, (_, a) in methods.items() if a}
    for name, (params, _) in methods.items():
        assert callable(getattr(B, name, None)), f"B200Backend lacks {name}"
        ours = [p.name for p in inspect.signature(getattr(B, name)).parameters.values()
                if p.kind in (p.POSITIONAL_ONLY, p.POSITIONAL_OR_KEYWORD)][1:]
        assert ours[:len(params)] == params, (name, ours, params)
        extra = [p for p in inspect.signature(getattr(B, name)).parameters.values()
                 if p.name not in params and p.name != "self"]
        assert all(p.default is not p.empty or p.kind in (p.VAR_POSITIONAL, p.VAR_KEYWORD) for p in extra), name
    # the constructor takes (ops, flow, opts) positionally, like every reference backend
    init = [p.name for p in inspect.signature(B.__init__).parameters.values()
            if p.kind == p.POSITIONAL_OR_KEYWORD][1:]
    assert init == ["ops", "flow", "opts"]


def test_every_attribute_the_reference_sets_or_callers_read_exists():
    ours = _our_attributes()
    missing = sorted(_init_attributes(_backend_class()) - ours)
    assert not missing, f"attributes the reference's Backend sets but B200Backend lacks: {missing}"
    used = set()
    for rel in CALLERS:
        for node in ast.walk(_tree(rel)):
            if isinstance(node, ast.Attribute) and isinstance(node.value, ast.Name) and node.value.id in BACKEND_NAMES:
                used.add(node.attr)
    assert {"run", "scheme", "asarray", "to_numpy", "limiter_activity", "n_mean_repaired"} <= used
    missing = sorted(used - ours)
    assert not missing, f"attributes the reference's callers read off a backend but B200Backend lacks: {missing}"
