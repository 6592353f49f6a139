"""CPU checks of the C-ABI boundary: the library loads without a GPU and
exports every entry point that include/*.h declares; record layouts match the
host mirrors."""

import ctypes
import glob
import os
import re

import numpy as np

import apgar_b200
from apgar_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for header in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(header).read()
        names.update(re.findall(r"APGAR_B200_API\s+[\w\s\*]+?\b(apgar_b200_\w+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_entry_point():
    lib = apgar_b200.lib()
    names = declared_symbols()
    assert len(names) >= 12
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert lib.apgar_b200_abi_version() == 1


def test_record_layouts():
    assert synth.NET_DTYPE.itemsize == 40
    assert apgar_b200.RESULT_DTYPE.itemsize == 48
    assert ctypes.sizeof(apgar_b200.PlanInfo) == 40


def test_last_error_roundtrip_without_gpu():
    lib = apgar_b200.lib()
    # a null-argument call fails on the host before touching CUDA
    rc = lib.apgar_b200_lattice_upload(None, None)
    assert rc == 4
    buf = ctypes.create_string_buffer(256)
    n = lib.apgar_b200_last_error(buf, ctypes.c_size_t(256))
    assert n > 0 and b"null" in buf.value


def test_python_mirror_never_imports_the_oracle():
    for path in glob.glob(os.path.join(ROOT, "apgar_b200", "**", "*.py"), recursive=True):
        text = open(path).read()
        assert "import oracle" not in text and "from oracle" not in text, path


def test_view_upload_rejects_corrupt_views_without_gpu():
    """Upload validation runs on the host before any device call."""
    from apgar_b200 import dropin
    from tests.golden import ref_corpus

    case = ref_corpus.load_case(ref_corpus.HERE + "/dense_corridors.bin")
    nodes = case.nodes.copy()
    nodes["neighbors"][0][0], nodes["neighbors"][0][1] = nodes["neighbors"][0][1], nodes["neighbors"][0][0]
    nodes["legal_edges"][0] |= 0x3
    try:
        dropin.View(case.header, case.layers, nodes, case.runs, case.run_nodes)
    except apgar_b200.BackendError as e:
        assert e.code == 4 and "upload rejected" in e.detail
    else:
        raise AssertionError("corrupt view accepted")


def test_new_entry_points_refuse_null_handles_on_the_host():
    """Each refuses a null handle or argument with INTERNAL_INVARIANT (4) and a
    'null' detail, before any device call."""
    lib = apgar_b200.lib()
    calls = [
        lambda: lib.apgar_b200_lattice_validate(None, None, ctypes.c_uint32(1), None, None,
                                                ctypes.c_uint64(0), None),
        lambda: lib.apgar_b200_confirm_disconnected(None, None, ctypes.c_uint32(1), None,
                                                    ctypes.c_uint64(0), None, None),
        lambda: lib.apgar_b200_validate_predecessors(None, None, ctypes.c_uint32(1), None,
                                                     ctypes.c_uint64(0), None, None, None, None),
        lambda: lib.apgar_b200_negotiation_set_usage_buffer(None, None),
    ]
    buf = ctypes.create_string_buffer(256)
    for call in calls:
        assert call() == 4
        lib.apgar_b200_last_error(buf, ctypes.c_size_t(256))
        assert b"null" in buf.value, buf.value
    # a negotiation step without a negotiation, and with an unknown phase
    assert lib.apgar_b200_negotiation_step(None, ctypes.c_uint32(0), ctypes.c_uint32(0),
                                           ctypes.c_uint32(0), None) == 4
