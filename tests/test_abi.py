"""CPU: the C-ABI library loads, exports every entry point the header declares,
its struct layouts match the ctypes mirror, and its host-side mesh set-up
agrees with the oracle's independent restatement."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

import oracle as O
import theseus_b200 as T
from theseus_b200._abi import Config, Geometry

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))
           if f.endswith(".h")]


def declared_functions():
    names = set()
    for h in HEADERS:
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names.update(re.findall(r"\b(thx_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = T.library()
    names = declared_functions()
    assert len(names) >= 12
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_struct_layout_matches_header():
    src = r'''
#include <stdio.h>
#include <stddef.h>
#include "theseus_b200.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu\n", sizeof(thx_config), offsetof(thx_config, gamma),
         offsetof(thx_config, modal_threshold), sizeof(thx_geometry), offsetof(thx_geometry, face_wplus));
  return 0;
}
'''
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        open(c, "w").write(src)
        exe = os.path.join(d, "t")
        subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe])
        got = [int(x) for x in subprocess.check_output([exe]).split()]
    want = [C.sizeof(Config), Config.gamma.offset, Config.modal_threshold.offset,
            C.sizeof(Geometry), Geometry.face_wplus.offset]
    assert got == want


@pytest.mark.parametrize("dim,order,n", [(2, 3, (4, 3)), (3, 4, (2, 3, 2)), (3, 2, (1, 2, 3))])
def test_box_geometry_matches_oracle(dim, order, n):
    lo, hi = [-1.0, 0.5, 2.0][:dim], [1.5, 2.0, 3.0][:dim]
    a = T.periodic_box(dim, order, n, lo, hi)
    b = O.box_mesh(dim, order, n, lo, hi)
    for k in ("jac", "metric", "face_normal", "face_wminus", "face_wplus", "coords"):
        assert np.allclose(getattr(a, k), getattr(b, k), rtol=1e-15, atol=1e-15), k
    assert np.array_equal(a.face_elem, b.face_elem)
    assert np.array_equal(a.face_lface, b.face_lface)


def test_lgl_rule():
    for np_ in range(2, 9):
        x, w = T.lgl(np_)
        assert abs(w.sum() - 1.0) < 1e-14
        xo, wo, *_ = O.operators(np_ - 1)
        assert np.allclose(x, xo, atol=1e-15) and np.allclose(w, wo, atol=1e-15)
        # exact for polynomials of degree 2*np-3
        k = 2 * np_ - 3
        assert abs((w * x ** k).sum() - 1.0 / (k + 1)) < 1e-13


def test_selection_strings():
    from theseus_b200._abi import flux_id
    assert flux_id("Chandrashekar") == 0 and flux_id("chan") == 0
    assert flux_id("ranocha") == 1 and flux_id("PiFlux") == 2 and flux_id("hll") == 3
    assert flux_id("LFR") == 4 and flux_id("lax_friedrichs") == 4 and flux_id("roe") == 5
    with pytest.raises(ValueError):
        flux_id("godunov")


def test_no_cpu_fallback():
    """Without a GPU the operator refuses to run instead of falling back."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    m = T.periodic_box(2, 3, (2, 2), [0, 0], [1, 1])
    h = C.c_void_p()
    cfg = T.make_config()
    st = T.library().thx_create(C.byref(m.struct()), C.byref(cfg), C.byref(h))
    assert st == 4  # THX_ERR_NO_DEVICE
    with pytest.raises(T.THXError):
        T.EulerOperator(m)


def test_invalid_arguments():
    lib = T.library()
    h = C.c_void_p()
    assert lib.thx_create(None, None, C.byref(h)) == 1
    m = T.periodic_box(2, 9, (2, 2), [0, 0], [1, 1])  # p=9: not instantiated
    cfg = T.make_config()
    st = lib.thx_create(C.byref(m.struct()), C.byref(cfg), C.byref(h))
    assert st in (2, 4)
    assert lib.thx_rhs(None, None, None, None) == 1
