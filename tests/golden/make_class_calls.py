"""Records the backend calls that the reference's own class code makes and
the oracle's results of them: tests/golden/class_calls.npz.

    python tests/golden/make_class_calls.py      (in the container holding
                                                  the reference source tree)

The reference's class modules (pyshtools/shclasses/shcoeffs.py, shgrid.py),
its backend registry (pyshtools/backends/backends.py) and its expand and
rotate packages with their backend injectors (pyshtools/expand/__init__.py,
pyshtools/rotate/__init__.py) are imported from the source tree; what they
import beyond numpy and scipy (matplotlib, xarray, boule, the compiled
Fortran backend, the I/O and spectral-analysis packages, the Legendre
module) is replaced by stand-ins that the transform path never calls.  The
'cuda' entry of the registry is a recorder: each call the classes make
(SHCoeffs.expand -> MakeGridDH / MakeGridGLQ, SHGrid.expand -> SHExpandDH /
SHExpandGLQ) is stored with its array inputs and keyword arguments, and is
answered by the oracle.  The GPU test replays these calls through
shtools_b200.backend and compares with the stored oracle outputs.

The reference tree is read only by this script and by the CPU test that
checks the registration and the injectors (tests/test_reference_classes.py);
its location is the environment variable SHTC_REFERENCE, by default
/root/reference.
"""
import importlib.util
import json
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF_ROOT = os.environ.get("SHTC_REFERENCE", "/root/reference")
OUT = os.path.join(HERE, "class_calls.npz")


def _module(name, **attrs):
    m = types.ModuleType(name)
    m.__dict__.update(attrs)
    sys.modules[name] = m
    return m


def _package(name, path):
    m = _module(name)
    m.__path__ = [path]
    return m


def _load(name, path):
    spec = importlib.util.spec_from_file_location(name, path)
    m = importlib.util.module_from_spec(spec)
    sys.modules[name] = m
    spec.loader.exec_module(m)
    return m


def _unused(name):
    def f(*a, **k):
        raise NotImplementedError("%s is not on the transform path" % name)
    f.__name__ = name
    return f


# names the reference's packages import from its compiled backend
_SHTOOLS_NAMES = [
    "GLQGridCoord", "SHExpandLSQ", "SHExpandLSQ_G", "SHExpandWLSQ", "SHExpandWLSQ_G",
    "LSQ_G", "MakeGrid2D", "MakeGridPoint", "MakeGridPointC", "SHMultiply", "djpi2",
    "SHRotateCoef", "SHRotateRealCoef", "SHExpandGLQ", "SHExpandGLQC", "SHExpandDH",
    "SHExpandDHC", "MakeGridGLQ", "MakeGridGLQC", "MakeGridDH", "MakeGridDHC",
    "MakeGradientDH",
]


def load_reference(ref_root=REF_ROOT):
    """Imports the reference's class modules, backend registry and
    injectors with stand-ins for their other imports.  Returns a namespace
    with the modules: shcoeffs, shgrid, backends (the registry), expand,
    rotate, shtools (the stand-in of the compiled backend)."""
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    pkg = os.path.join(ref_root, "pyshtools")
    if not os.path.isdir(os.path.join(pkg, "shclasses")):
        raise FileNotFoundError("no reference source tree at %s" % ref_root)
    for k in [k for k in sys.modules if k == "pyshtools" or k.startswith("pyshtools.")]:
        del sys.modules[k]
    # plotting and data libraries imported at module level by the classes
    mpl = _module("matplotlib")
    mpl.pyplot = _module("matplotlib.pyplot")
    _module("mpl_toolkits")
    _module("mpl_toolkits.axes_grid1", make_axes_locatable=_unused("make_axes_locatable"))
    _module("xarray")
    _module("boule", Sphere=object, Ellipsoid=object, TriaxialEllipsoid=object)
    _package("pyshtools", pkg)
    _package("pyshtools.backends", os.path.join(pkg, "backends"))
    shtools = _module("pyshtools.backends.shtools",
                      **{n: _unused(n) for n in _SHTOOLS_NAMES})
    shtools.SHGLQ = O.shglq
    _module("pyshtools.backends.ducc0_wrapper", available=lambda: False,
            set_nthreads=_unused("set_nthreads"))
    backends = _load("pyshtools.backends.backends", os.path.join(pkg, "backends", "backends.py"))
    b = sys.modules["pyshtools.backends"]
    for n in ("select_preferred_backend", "preferred_backend", "preferred_backend_module",
              "backend_module"):
        setattr(b, n, getattr(backends, n))
    b.shtools = shtools
    _module("pyshtools.legendre", legendre=_unused("legendre"))
    expand = _load("pyshtools.expand", os.path.join(pkg, "expand", "__init__.py"))
    rotate = _load("pyshtools.rotate", os.path.join(pkg, "rotate", "__init__.py"))
    _module("pyshtools.spectralanalysis", spectrum=_unused("spectrum"),
            cross_spectrum=_unused("cross_spectrum"))
    _module("pyshtools.shio", **{n: _unused(n) for n in (
        "convert", "shread", "shwrite", "read_dov", "write_dov", "read_bshc", "write_bshc")})
    _package("pyshtools.shclasses", os.path.join(pkg, "shclasses"))
    shgrid = _load("pyshtools.shclasses.shgrid", os.path.join(pkg, "shclasses", "shgrid.py"))
    shcoeffs = _load("pyshtools.shclasses.shcoeffs",
                     os.path.join(pkg, "shclasses", "shcoeffs.py"))
    return types.SimpleNamespace(shcoeffs=shcoeffs, shgrid=shgrid, backends=backends,
                                 expand=expand, rotate=rotate, shtools=shtools)


class Recorder(types.ModuleType):
    """The 'cuda' registry entry while recording: the four real transforms
    store their inputs and keywords and are answered by the oracle."""

    def __init__(self):
        super().__init__("recorder")
        from oracle import oracle as O
        self.O = O
        self.calls = []
        for n in ("SHExpandGLQC", "SHExpandDHC", "MakeGridGLQC", "MakeGridDHC",
                  "MakeGradientDH", "SHRotateRealCoef"):
            setattr(self, n, _unused(n))

    def _rec(self, name, arrays, kwargs, out):
        self.calls.append((name, [np.array(a, dtype=np.float64) for a in arrays],
                           dict(kwargs), np.array(out)))
        return out

    def MakeGridDH(self, cilm, lmax=None, norm=1, sampling=1, csphase=1, lmax_calc=None,
                   extend=False):
        kw = dict(lmax=lmax, norm=norm, sampling=sampling, csphase=csphase,
                  lmax_calc=lmax_calc, extend=bool(extend))
        out = self.O.makegrid_dh(cilm, lmax=lmax, norm=norm, sampling=sampling,
                                 csphase=csphase, lmax_calc=lmax_calc, extend=int(bool(extend)))
        return self._rec("MakeGridDH", [cilm], kw, out)

    def SHExpandDH(self, griddh, norm=1, sampling=1, csphase=1, lmax_calc=None):
        kw = dict(norm=norm, sampling=sampling, csphase=csphase, lmax_calc=lmax_calc)
        out = self.O.shexpand_dh(np.ascontiguousarray(griddh), norm=norm, sampling=sampling,
                                 csphase=csphase, lmax_calc=lmax_calc)
        return self._rec("SHExpandDH", [griddh], kw, out)

    def MakeGridGLQ(self, cilm, zero=None, lmax=None, norm=1, csphase=1, lmax_calc=None,
                    extend=False):
        kw = dict(lmax=lmax, norm=norm, csphase=csphase, lmax_calc=lmax_calc,
                  extend=bool(extend))
        L = lmax if lmax is not None else np.shape(cilm)[1] - 1
        z = zero if zero is not None else self.O.shglq(L)[0]
        out = self.O.makegrid_glq(cilm, zero=z, lmax=lmax, norm=norm, csphase=csphase,
                                  lmax_calc=lmax_calc, extend=int(bool(extend)))
        arrays = [cilm] if zero is None else [cilm, zero]
        if zero is not None:
            kw["zero"] = "array"
        return self._rec("MakeGridGLQ", arrays, kw, out)

    def SHExpandGLQ(self, gridglq, w=None, zero=None, norm=1, csphase=1, lmax_calc=None):
        kw = dict(norm=norm, csphase=csphase, lmax_calc=lmax_calc)
        out = self.O.shexpand_glq(np.ascontiguousarray(gridglq), w=w, zero=zero, norm=norm,
                                  csphase=csphase, lmax_calc=lmax_calc)
        return self._rec("SHExpandGLQ", [gridglq, w, zero], kw, out)


def cases(R, O):
    """The class-level round trips; each returns the final coefficients."""
    SHCoeffs = R.shcoeffs.SHCoeffs

    def dh_4pi():
        c = SHCoeffs.from_array(O.power_law_cilm(31, 8101), normalization="4pi", csphase=1)
        g = c.expand(grid="DH", extend=False, backend="cuda")
        return g.expand(backend="cuda").coeffs

    def dh2_ortho_padded():
        c = SHCoeffs.from_array(O.power_law_cilm(40, 8102), normalization="ortho",
                                csphase=-1)
        g = c.expand(grid="DH2", lmax=48, lmax_calc=30, extend=True, backend="cuda")
        return g.expand(normalization="ortho", csphase=-1, lmax_calc=20,
                        backend="cuda").coeffs

    def glq_schmidt():
        c = SHCoeffs.from_array(O.power_law_cilm(50, 8103), normalization="schmidt")
        g = c.expand(grid="GLQ", extend=True, backend="cuda")
        return g.expand(normalization="schmidt", backend="cuda").coeffs

    def dh2_unnorm():
        c = SHCoeffs.from_array(O.power_law_cilm(12, 8104), normalization="unnorm")
        g = c.expand(grid="DH2", backend="cuda")
        return g.expand(normalization="unnorm", backend="cuda").coeffs

    def preferred_dh2():
        # through the preferred backend, as after select_preferred_backend('cuda')
        c = SHCoeffs.from_array(O.power_law_cilm(24, 8105))
        g = c.expand()
        return g.expand().coeffs

    return [("dh_4pi", dh_4pi), ("dh2_ortho_padded", dh2_ortho_padded),
            ("glq_schmidt", glq_schmidt), ("dh2_unnorm", dh2_unnorm),
            ("preferred_dh2", preferred_dh2)]


def record(ref_root=REF_ROOT):
    """Runs the cases through the recorder; returns {case: (calls, coeffs)}."""
    R = load_reference(ref_root)
    from oracle import oracle as O
    rec = Recorder()
    R.backends._available_backends["cuda"] = rec
    R.backends.select_preferred_backend("cuda")
    out = {}
    for name, fn in cases(R, O):
        rec.calls = []
        coeffs = fn()
        out[name] = (list(rec.calls), np.array(coeffs))
    R.backends.select_preferred_backend("shtools")
    return out


def main():
    res = record()
    arrays, index = {}, {}
    for case, (calls, coeffs) in res.items():
        entries = []
        for i, (fname, args, kw, out) in enumerate(calls):
            keys = []
            for j, a in enumerate(args):
                k = "%s_%d_in%d" % (case, i, j)
                arrays[k] = a
                keys.append(k)
            arrays["%s_%d_out" % (case, i)] = out
            entries.append({"function": fname, "inputs": keys, "kwargs": kw,
                            "output": "%s_%d_out" % (case, i)})
        arrays["%s_coeffs" % case] = coeffs
        index[case] = entries
    arrays["index"] = np.frombuffer(json.dumps(index, sort_keys=True).encode(), dtype=np.uint8)
    np.savez_compressed(OUT, **arrays)
    print("wrote %s: %d cases, %d calls" % (OUT, len(index),
                                            sum(len(v) for v in index.values())))


if __name__ == "__main__":
    main()
