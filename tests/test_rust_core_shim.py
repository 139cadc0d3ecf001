"""propaq_b200.rust_core against the reference's compiled-module surface
(propaq/_rust_core/__init__.pyi, read as text from the reference tree; the tests
skip when it is absent).

* Every name the stub exports exists in the shim.
* For the numerical path's classes, every method, property and constructor of
  the stub exists with the same parameter names in the same order and the
  same defaults present.
* The out-of-scope names (surrogate propagators and models, the hybrid MPS
  expectation) raise NotImplementedError when used.
* With the shim installed as propaq._rust_core, the reference's own
  pure-Python modules import unchanged (extrapolators, noise, truncation,
  propagator base classes, log parser) and build their objects from the
  shim's classes."""

from __future__ import annotations

import ast
import importlib
import inspect
import sys
import types

import pytest
from conftest import REFERENCE_TREE

from propaq_b200 import rust_core

STUB = REFERENCE_TREE / "propaq" / "_rust_core" / "__init__.pyi"
OUTSIDE = {"MajoranaSurrogateModel", "MajoranaSurrogatePropagator", "PauliSurrogateModel",
           "PauliSurrogatePropagator", "hybrid_expectation"}


def stub_tree():
    if not STUB.exists():
        pytest.skip("the reference tree is not present")
    return ast.parse(STUB.read_text())


def stub_all(tree):
    for node in tree.body:
        if isinstance(node, ast.Assign) and node.targets[0].id == "__all__":
            return [e.value for e in node.value.elts]
    raise AssertionError("no __all__ in the stub")


def stub_classes(tree):
    return {n.name: n for n in tree.body if isinstance(n, ast.ClassDef)}


def params_of(fn: ast.FunctionDef):
    """(names, names with defaults) of a stub method, without self / cls."""
    a = fn.args
    names = [x.arg for x in a.posonlyargs + a.args][1:] + [x.arg for x in a.kwonlyargs]
    pos = [x.arg for x in a.posonlyargs + a.args][1:]
    with_default = set(pos[len(pos) - len(a.defaults):]) if a.defaults else set()
    with_default |= {x.arg for x, d in zip(a.kwonlyargs, a.kw_defaults) if d is not None}
    return names, with_default


def shim_params(obj):
    sig = inspect.signature(obj)
    ps = [p for p in sig.parameters.values() if p.kind not in (p.VAR_POSITIONAL, p.VAR_KEYWORD)]
    if ps and ps[0].name in ("self", "cls"):
        ps = ps[1:]
    return [p.name for p in ps], {p.name for p in ps if p.default is not p.empty}


def test_every_stub_name_exists():
    tree = stub_tree()
    missing = [n for n in stub_all(tree) if not hasattr(rust_core, n)]
    assert not missing, missing


# An instance of each numerical class, for the stub's properties (which are
# instance attributes here).
def _instances():
    r = rust_core
    return {
        "CoefficientTruncator": r.CoefficientTruncator(1e-3), "FrequencyTruncationPolicy": r.FrequencyTruncationPolicy(),
        "FrequencyTruncator": r.FrequencyTruncator(3), "Logger": r.Logger("run.jsonl"),
        "PropagationResult": r.PropagationResult(0.5, [1, 2]), "Simplify": r.Simplify(),
        "TermBudget": r.TermBudget(10), "TruncationPolicy": r.TruncationPolicy(3, 1e-4),
        "UniformNoiseModel": r.UniformNoiseModel(0.1), "WeightTruncator": r.WeightTruncator(4),
        "MajoranaMonomial": r.MajoranaMonomial(0b11, 4), "PauliString": r.PauliString(1, 2, 3),
        "PauliTermSum": r.PauliTermSum(), "MajoranaTermSum": r.MajoranaTermSum(),
        "PauliPropagator": r.PauliPropagator(), "MajoranaPropagator": r.MajoranaPropagator(),
    }


def _same_params(got, got_def, want, want_def):
    """Same names in the same order (a leading underscore, which the stub uses
    for unused arguments, aside); extra trailing parameters with defaults are
    allowed; every stub default is a default here."""
    strip = lambda xs: [x.lstrip("_") for x in xs]  # noqa: E731
    g, w = strip(got), strip(want)
    if g[:len(w)] != w or any(x not in got_def for x in got[len(w):]):
        return False
    return set(strip(want_def)) <= set(strip(got_def))


def test_numerical_classes_match_the_stub():
    tree = stub_tree()
    inst = _instances()
    problems = []
    dunder = ("__repr__", "__hash__", "__eq__", "__len__", "__iter__", "__next__", "__setitem__", "__getitem__",
              "__matmul__")
    for name, cls in stub_classes(tree).items():
        if name in OUTSIDE:
            continue
        ours = getattr(rust_core, name)
        for fn in (n for n in cls.body if isinstance(n, ast.FunctionDef)):
            deco = [d.id if isinstance(d, ast.Name) else getattr(d, "attr", "") for d in fn.decorator_list]
            if "property" in deco or "setter" in deco:
                obj = inst.get(name)
                as_property = isinstance(inspect.getattr_static(ours, fn.name, None), property)
                if not as_property and (obj is None or not hasattr(obj, fn.name)):
                    problems.append(f"{name}.{fn.name} (property) missing")
                continue
            if fn.name in dunder:
                if not hasattr(ours, fn.name):
                    problems.append(f"{name}.{fn.name} missing")
                continue
            target = ours.__init__ if fn.name == "__new__" else inspect.getattr_static(ours, fn.name, None)
            if target is None:
                problems.append(f"{name}.{fn.name} missing")
                continue
            want, want_def = params_of(fn)
            if "staticmethod" in deco:  # no self in the stub's list
                a = fn.args
                want = [x.arg for x in a.posonlyargs + a.args]
                pos = want
                want_def = set(pos[len(pos) - len(a.defaults):]) if a.defaults else set()
            if isinstance(target, (staticmethod, classmethod)):
                target = target.__func__
            got, got_def = shim_params(target)
            if not _same_params(got, got_def, want, want_def):
                problems.append(f"{name}.{fn.name}: parameters {got} (defaults {sorted(got_def)}) vs stub {want} "
                                f"(defaults {sorted(want_def)})")
    assert not problems, "\n".join(problems)


def test_outside_names_refuse():
    for name in ("PauliSurrogatePropagator", "MajoranaSurrogatePropagator", "PauliSurrogateModel",
                 "MajoranaSurrogateModel"):
        with pytest.raises(NotImplementedError):
            getattr(rust_core, name)()
    with pytest.raises(NotImplementedError):
        rust_core.hybrid_expectation(None, [])
    assert rust_core.rust_available()


@pytest.fixture
def reference_package():
    """The reference's propaq package (its pure-Python modules, unchanged) with
    the shim as propaq._rust_core.  propaq/__init__.py itself is not run: it
    reads the installed distribution's metadata and imports the Qiskit front
    end; the submodules are imported directly."""
    if not (REFERENCE_TREE / "propaq").is_dir():
        pytest.skip("the reference tree is not present")
    ours = ("propaq", "qiskit")
    mine = lambda k: k in ours or k.split(".")[0] in ours  # noqa: E731
    saved = {k: v for k, v in sys.modules.items() if mine(k)}
    for k in saved:
        del sys.modules[k]
    _placeholder_qiskit()
    pkg = types.ModuleType("propaq")
    pkg.__path__ = [str(REFERENCE_TREE / "propaq")]
    sys.modules["propaq"] = pkg
    rust_core.install()
    yield pkg
    for k in [k for k in sys.modules if mine(k)]:
        del sys.modules[k]
    sys.modules.update(saved)


def _placeholder_qiskit():
    """Qiskit is not in this image.  The reference's datatypes and circuits
    name a few of its classes at import time only (isinstance checks and
    converters the numerical path does not call); empty stand-ins let those
    modules import."""
    names = {"qiskit": ["QuantumCircuit", "transpile"], "qiskit.circuit": ["Instruction", "Parameter"],
             "qiskit.circuit.parameterexpression": ["ParameterExpression"],
             "qiskit.quantum_info": ["SparsePauliOp"], "qiskit.converters": ["circuit_to_dag"]}
    for mod_name, attrs in names.items():
        mod = types.ModuleType(mod_name)
        mod.__path__ = []
        for a in attrs:
            setattr(mod, a, type(a, (), {}))
        sys.modules[mod_name] = mod
    for mod_name in names:
        if "." in mod_name:
            parent, child = mod_name.rsplit(".", 1)
            setattr(sys.modules[parent], child, sys.modules[mod_name])


@pytest.mark.parametrize("module", ["propaq.noise", "propaq.truncation", "propaq.log_parser",
                                    "propaq.extrapolators.zne", "propaq.extrapolators.zce"])
def test_reference_modules_import_on_the_shim(reference_package, module):
    mod = importlib.import_module(module)
    assert mod is not None
    assert sys.modules["propaq._rust_core"] is rust_core


def test_reference_extrapolator_builds_shim_objects(reference_package):
    zne = importlib.import_module("propaq.extrapolators.zne")
    ext = zne.ZeroNoiseExtrapolator(lambda x, a, b: a + b * x, [0.01, 0.02])
    built = ext.build_noise(0.05)
    assert isinstance(built, rust_core.UniformNoiseModel) and built.damping == 0.05
    zce = importlib.import_module("propaq.extrapolators.zce")
    # the reference subclasses the compiled classes (propaq/truncation/__init__.py:15-40);
    # its truncators are accepted by the engine's propagators
    assert issubclass(zce.WeightTruncator, rust_core.WeightTruncator)
    prop = rust_core.PauliPropagator(truncation=[zce.WeightTruncator(4), zce.CoefficientTruncator(1e-3)])
    assert [type(t).__name__ for t in prop.truncators] == ["WeightTruncator", "CoefficientTruncator"]
