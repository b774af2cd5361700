"""libccs on the CPU: it loads, exports every entry point include/ccs.h declares, and its host-side
constants and errors behave like the reference's (no GPU work here)."""

from __future__ import annotations

import re

import numpy as np
import pytest

from conftest import ROOT
from cuda_cube_solver import coords, kinds, native


def _declared() -> set[str]:
    text = (ROOT / "include" / "ccs.h").read_text()
    return set(re.findall(r"^(?:int|const char\*)\s+(ccs_\w+)\(", text, re.M))


def test_every_declared_symbol_is_exported():
    declared = _declared()
    assert len(declared) >= 20
    for name in declared:
        assert hasattr(native.lib, name), name
    assert set(native.EXPORTED) == declared


def test_kind_constants_match_host_model():
    cc = coords.corner_classes()
    for name in ["304", "s4", "d4f", "a4t", "d4t", "d4", "a4"]:
        t = native.kind_tables(name)
        assert np.array_equal(t["classidx"], cc.classidx)
        assert np.array_equal(t["class_rep"], cc.rep)
        assert np.array_equal(t["class_stab"], cc.stab)
        nec, n = native.kind_info(name)
        assert n == kinds.N_CLASSES * kinds.get(name).n_edge
        if name != "304":
            k = kinds.get(name)
            assert nec == k.nec
            assert np.array_equal(t["gen_class"], k.gen[0]) and np.array_equal(t["gen_rep"], k.gen[1])


def test_unknown_kind_is_an_argument_error():
    with pytest.raises(native.CcsError) as exc:
        native.kind_info("nope")
    assert exc.value.code == native.CCS_E_ARG
    assert "unknown table kind" in str(exc.value)


def test_custom_group_kind_registration():
    gens = kinds.GROUP_KINDS["d4t"]
    native.register_group_kind("mine-d4t", gens)
    t = native.kind_tables("mine-d4t")
    assert np.array_equal(t["gen_class"], kinds.get("d4t").gen[0])
    with pytest.raises(native.CcsError, match="not normalised"):
        native.register_group_kind("swap01", [((1, 0, 2, 3), (0, 0, 0, 0))])


def test_noalloc_limit_matches_header():
    text = (ROOT / "include" / "ccs.h").read_text()
    assert f"#define CCS_NOALLOC_MAX_CUBES {native.NOALLOC_MAX_CUBES}" in text
