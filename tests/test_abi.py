"""The C-ABI library loads and exports every entry point include/epp.h declares; the ctypes
mirror matches the header (no GPU needed)."""
import ctypes as C
import os
import re
import subprocess

import pytest

from epp import abi
from epp import lib as epplib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "epp.h")


def header_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int32_t|const char\*|void)\s+(epp_\w+)\s*\(", text, re.M)))


def test_header_functions_exported():
    names = header_functions()
    assert len(names) >= 15
    out = subprocess.check_output(["nm", "-D", "--defined-only", epplib.LIB_PATH]).decode()
    exported = set(re.findall(r"\bT (epp_\w+)", out))
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    assert set(names) == set(epplib.EXPORTS)


def test_library_loads_without_gpu():
    lib = epplib.load()
    assert lib.epp_abi_version() == abi.EPP_ABI_VERSION
    n = C.c_int32(-1)
    rc = lib.epp_device_count(C.byref(n))
    assert rc in (abi.EPP_OK, abi.EPP_ERR_NO_DEVICE)


def test_struct_sizes_match_header(tmp_path):
    """Compile a tiny C probe against include/epp.h and compare sizeof/offsetof with ctypes."""
    src = r'''
#include <stdio.h>
#include <stddef.h>
#include "epp.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu\n", sizeof(epp_domain), sizeof(epp_physics), sizeof(epp_config),
         sizeof(epp_column_map), sizeof(epp_integrals), offsetof(epp_config, hbm_budget_bytes));
  return 0;
}
'''
    tmp = str(tmp_path)
    with open(os.path.join(tmp, "p.c"), "w") as f:
        f.write(src)
    exe = os.path.join(tmp, "p")
    subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), "-o", exe, os.path.join(tmp, "p.c")])
    vals = [int(v) for v in subprocess.check_output([exe]).split()]
    assert vals == [C.sizeof(abi.epp_domain), C.sizeof(abi.epp_physics), C.sizeof(abi.epp_config),
                    C.sizeof(abi.epp_column_map), C.sizeof(abi.epp_integrals),
                    abi.epp_config.hbm_budget_bytes.offset]


def test_create_fails_loudly_without_gpu():
    """No CPU fallback: without a device the context cannot be created."""
    lib = epplib.load()
    n = C.c_int32(0)
    if lib.epp_device_count(C.byref(n)) == abi.EPP_OK:
        pytest.skip("a GPU is present")
    d = abi.make_domain(2, 0.1, [0, 0], [1, 1])
    cfg = abi.make_config(d, 10, [[1]])
    with pytest.raises(epplib.EppError):
        epplib.Context(cfg)


def test_context_bytes_capacity_limit():
    """epp_context_bytes is host arithmetic (no device): the footprint grows with the capacity,
    and capacities above 2^28 are refused (neighbour-list entries hold 28-bit indices)."""
    d = abi.make_domain(2, 0.006, [-0.02, -0.02], [4.02, 3.02])
    small = epplib.context_bytes(abi.make_config(d, 100000, [[1, 1], [1, 0]]))
    large = epplib.context_bytes(abi.make_config(d, 1000000, [[1, 1], [1, 0]]))
    assert 0 < small < large
    with pytest.raises(epplib.EppError) as e:
        epplib.context_bytes(abi.make_config(d, (1 << 28) + 1, [[1, 1], [1, 0]]))
    assert e.value.code == abi.EPP_ERR_CAPACITY
