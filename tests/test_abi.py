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
