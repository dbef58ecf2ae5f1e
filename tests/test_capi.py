"""The C ABI library without a GPU: it loads, exports every entry point
include/sbk.h declares, validates materials and rules as the reference's
Material::set_plasticity does, and refuses compute calls without a device
(no CPU fallback)."""
from __future__ import annotations

import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "sbk.h")).read()
    return sorted(set(re.findall(r"^(?:int|const char\*)\s+(sbk_\w+)\s*\(", text, flags=re.M)))


def test_library_exports_every_declared_symbol(pkg):
    lib = ctypes.CDLL(pkg.library_path())
    names = declared_symbols()
    assert len(names) >= 28
    for name in names:
        assert hasattr(lib, name), name
    # ... and the bindings cover them all.
    assert set(names) == set(pkg._capi.SIGNATURES)


def test_rule_sizes(pkg):
    m = pkg.material
    assert m.rule_size(2, 0, 2) == 8
    assert m.rule_size(2, 5, 2) == 20
    assert m.rule_size(3, 0, 2) == 27
    assert m.rule_size(5, 0, 2) == 0  # in-plane orders 1 to 4 only
    assert m.rule_size(2, 8, 2) == 0  # through the thickness 1 to 7


def test_state_fields(pkg):
    m = pkg.material
    assert m.j2_steel().state_fields == 14
    assert m.hill_chaboche_sheet().state_fields == 26
    c = m.hill_chaboche_sheet().to_c()
    assert pkg._capi.lib().sbk_state_fields(ctypes.byref(c)) == 26


@pytest.mark.parametrize("law", ["hill_sheet", "hill_chaboche_sheet", "j2_steel"])
def test_yield_matrix_matches_oracle(pkg, orc, law):
    mat = getattr(pkg.material, law)()
    p = pkg.material.yield_matrix(mat)
    q = orc.yield_matrix(mat.as_dict())
    np.testing.assert_allclose(p, q, rtol=1e-14, atol=1e-14)


def test_invalid_material_is_refused(pkg):
    import dataclasses

    bad = dataclasses.replace(pkg.material.j2_steel(), poisson_ratio=0.5)
    with pytest.raises(pkg.SbkError) as e:
        pkg.material.yield_matrix(bad)
    assert e.value.status == 2
    bad = dataclasses.replace(pkg.material.hill_sheet(), r0=-1.0)
    with pytest.raises(pkg.SbkError):
        pkg.material.yield_matrix(bad)
    bad = pkg.Material(70e9, 0.3, yield_stress=0.0, hardening_modulus=1e9)
    with pytest.raises(pkg.SbkError):
        pkg.material.yield_matrix(bad)


def test_no_device_no_fallback(pkg):
    """Without a GPU the system refuses to be created (NO_EXTENSION)."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    mesh = pkg.structured_hex_mesh(2, 2, 1, 1.0, 1.0, 0.1)
    with pytest.raises(pkg.SbkError) as e:
        pkg.NonlinearSystem(mesh, pkg.material.j2_steel())
    assert e.value.status == 7
