"""The reference's class code on the 'cuda' backend, without a GPU.

tests/golden/class_calls.npz holds the backend calls that the reference's
own SHCoeffs.expand and SHGrid.expand make (pyshtools/shclasses/
shcoeffs.py:4325-4380, shgrid.py:2086-2115, 2992-3020) for DH, DH2 and GLQ
grids in the four normalisations, with the oracle's answers
(tests/golden/make_class_calls.py).  Here:
  * the fixture is pinned: the oracle reproduces every stored output, and
    each round trip's final coefficients are those of its last call;
  * every recorded call binds to the signature of shtools_b200.backend;
  * when the reference source tree is present (this container): the
    backend registers into the reference's own registry
    (pyshtools/backends/backends.py:27), select_preferred_backend('cuda')
    makes the reference's expand and rotate injectors
    (pyshtools/expand/__init__.py:91-111, pyshtools/rotate/__init__.py:18-21)
    bind this backend's functions, and the classes still make exactly the
    recorded calls.
tests/test_gpu_classes.py replays the calls on the GPU.
"""
import inspect
import json
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
FIXTURE = os.path.join(HERE, "golden", "class_calls.npz")


@pytest.fixture(autouse=True, scope="module")
def _drop_reference_modules():
    """The reference's modules and their stand-ins leave sys.modules with
    this file's tests."""
    before = set(sys.modules)
    yield
    for k in set(sys.modules) - before:
        if k.split(".")[0] in ("pyshtools", "matplotlib", "mpl_toolkits", "xarray", "boule",
                               "make_class_calls"):
            del sys.modules[k]


def _fixture():
    d = np.load(FIXTURE)
    return d, json.loads(bytes(d["index"]).decode())


def _oracle_call(O, fname, args, kw):
    kw = dict(kw)
    if fname == "MakeGridDH":
        kw["extend"] = int(kw["extend"])
        return O.makegrid_dh(args[0], **kw)
    if fname == "SHExpandDH":
        return O.shexpand_dh(args[0], **kw)
    if fname == "MakeGridGLQ":
        kw["extend"] = int(kw["extend"])
        kw.pop("zero", None)
        L = kw["lmax"] if kw.get("lmax") is not None else args[0].shape[1] - 1
        z = args[1] if len(args) > 1 else O.shglq(L)[0]
        return O.makegrid_glq(args[0], zero=z, **kw)
    if fname == "SHExpandGLQ":
        return O.shexpand_glq(args[0], w=args[1], zero=args[2], **kw)
    raise AssertionError(fname)


def test_fixture_reproduced_by_oracle(oracle):
    d, idx = _fixture()
    assert set(idx) == {"dh_4pi", "dh2_ortho_padded", "glq_schmidt", "dh2_unnorm",
                        "preferred_dh2"}
    for case, calls in idx.items():
        assert [c["function"][:4] for c in calls] == ["Make", "SHEx"]
        for c in calls:
            out = _oracle_call(oracle, c["function"], [d[k] for k in c["inputs"]], c["kwargs"])
            assert np.array_equal(out, d[c["output"]]), (case, c["function"])
        assert np.array_equal(d[calls[-1]["output"]], d[case + "_coeffs"])


def test_recorded_calls_bind_to_backend_signatures():
    from shtools_b200 import backend as B
    d, idx = _fixture()
    for case, calls in idx.items():
        for c in calls:
            kw = {k: v for k, v in c["kwargs"].items() if k != "zero"}
            args = [d[k] for k in c["inputs"]]
            if c["kwargs"].get("zero") == "array":
                kw["zero"] = args.pop(1)
            inspect.signature(getattr(B, c["function"])).bind(*args, **kw)


def _reference_or_skip():
    import make_class_calls as M
    if not os.path.isdir(os.path.join(M.REF_ROOT, "pyshtools", "shclasses")):
        pytest.skip("the reference source tree is not present")
    return M


def test_registry_and_injectors_of_the_reference():
    M = _reference_or_skip()
    from shtools_b200 import backend as B
    R = M.load_reference()
    reg = B.register(registry=R.backends)
    assert reg is R.backends
    assert R.backends.backend_module("cuda") is B
    R.backends.select_preferred_backend("cuda")
    try:
        assert R.backends.preferred_backend() == "cuda"
        for name in ("SHExpandGLQ", "SHExpandGLQC", "SHExpandDH", "SHExpandDHC",
                     "MakeGridGLQ", "MakeGridGLQC", "MakeGridDH", "MakeGridDHC",
                     "MakeGradientDH"):
            assert getattr(R.expand, name) is getattr(B, name), name
        assert R.rotate.SHRotateRealCoef is B.SHRotateRealCoef
    finally:
        R.backends.select_preferred_backend("shtools")
    assert R.expand.MakeGridDH is R.shtools.MakeGridDH


def test_classes_still_make_the_recorded_calls():
    M = _reference_or_skip()
    d, idx = _fixture()
    res = M.record()
    assert set(res) == set(idx)
    for case, (calls, coeffs) in res.items():
        assert len(calls) == len(idx[case])
        for (fname, args, kw, out), c in zip(calls, idx[case]):
            assert fname == c["function"] and kw == c["kwargs"], (case, fname)
            for a, k in zip(args, c["inputs"]):
                assert np.array_equal(a, d[k])
            assert np.array_equal(out, d[c["output"]])
        assert np.array_equal(coeffs, d[case + "_coeffs"])
