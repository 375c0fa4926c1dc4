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


@pytest.mark.parametrize("gap,first,last,code", [
    # 2^22 x 2^21 x 2^21 cells: the product is 2^64, which wraps to 0 in 64-bit arithmetic
    (1.0, [0, 0, 0], [4194304.0, 2097152.0, 2097152.0], abi.EPP_ERR_CAPACITY),
    # more than 2^31 cells on one axis: rejected before the conversion to int
    (1e-30, [0, 0, 0], [1.0, 1.0, 1.0], abi.EPP_ERR_CAPACITY),
    (float("nan"), [0, 0, 0], [1.0, 1.0, 1.0], abi.EPP_ERR_INVALID_ARGUMENT),
    (0.1, [0, 0, 0], [float("inf"), 1.0, 1.0], abi.EPP_ERR_CAPACITY),
    (0.1, [0, 0, 0], [0.05, 1.0, 1.0], abi.EPP_ERR_INVALID_ARGUMENT),   # no cell on the x axis
])
def test_domains_that_overflow_the_cell_count_are_refused(gap, first, last, code):
    """Both domain set-ups (the context's and the allocation-free cell sort's) check the cell
    count after every axis: a 3D domain whose cell count overflows 64 bits, or an axis beyond
    2^31 cells, is refused on the host, before anything is launched."""
    d = abi.make_domain(3, gap, first, last)
    with pytest.raises(epplib.EppError) as e:
        epplib.context_bytes(abi.make_config(d, 1000, [[1, 1], [1, 0]]))
    assert e.value.code == code
    lib = epplib.load()
    n_alive = C.c_int32(-1)
    rc = lib.epp_cell_sort_noalloc(C.byref(d), 10, C.c_void_p(16), None, None, C.c_void_p(16),
                                   C.byref(n_alive), None)
    assert rc == code
    assert n_alive.value == -1
