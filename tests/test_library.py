"""libccs on the CPU: it loads, exports every entry point include/ccs.h declares, and its host-side
constants and errors behave like the reference's (no GPU work here)."""

from __future__ import annotations

import ctypes
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


def _header_fields(struct: str) -> list[tuple[str, str]]:
    text = (ROOT / "include" / "ccs.h").read_text()
    body = re.search(r"typedef struct " + struct + r" \{(.*?)\} " + struct + ";", text, re.S).group(1)
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    return re.findall(r"^\s*(int|double|int32_t|uint32_t|uint64_t|uint8_t)\s+(\w+)(?:\[\d+\])?;", body, re.M)


def test_ctypes_structs_follow_the_header():
    """The Python bindings' structures have the header's fields in the header's order and types
    (the layout every FFI binding of ccs.h depends on)."""

    ct = {"int": ctypes.c_int, "double": ctypes.c_double, "int32_t": ctypes.c_int32, "uint32_t": ctypes.c_uint32,
          "uint64_t": ctypes.c_uint64}
    for struct, cls in (("ccs_solve_opts", native.SolveOpts), ("ccs_result", native.Result),
                        ("ccs_bfs_pass", native.BfsPass)):
        header = _header_fields(struct)
        fields = cls._fields_
        assert [n for _, n in header] == [n for n, _ in fields], struct
        for (ty, name), (_, cty) in zip(header, fields):
            if ty == "uint8_t":  # arrays of bytes
                assert issubclass(cty, ctypes.Array) and cty._type_ is ctypes.c_uint8, name
            elif issubclass(cty, ctypes.Array):
                assert cty._type_ is ct[ty], name
            else:
                assert cty is ct[ty], name
