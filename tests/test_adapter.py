"""The drop-in IPlanarRouteBackend shim (apgar_b200/adapter/) against the
reference's own interface.

CPU: the shim compiles against the reference headers, which also checks, by
static_assert, that every V1 record of the C ABI has the reference's size and
field offsets.  GPU: the native check drives the shim only through the
reference's interface types over every golden fixture case (goal labels
against the reference CPU A*, compact paths against the canonical
predecessor chain, the single-route pair)."""

import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BUILD = os.path.join(ROOT, "apgar_b200", "adapter", "build_adapter.sh")
CHECK = os.path.join(ROOT, "apgar_b200", "adapter", "_build", "adapter_check")


def test_shim_compiles_against_the_reference_interface():
    import oracle

    if oracle.reference_root() is None:
        pytest.skip("reference sources are absent (set APGAR_REFERENCE or run oracle/build_ref.sh)")
    out = subprocess.run(["bash", BUILD, "--check"], capture_output=True, text=True)
    assert out.returncode == 0, out.stderr[-2000:]


@pytest.mark.gpu
def test_shim_through_the_reference_interface_on_gpu():
    if not os.path.exists(CHECK):
        pytest.skip("native check not built (needs the reference headers at build time)")
    out = subprocess.run([CHECK, os.path.join(ROOT, "tests", "golden", "ref_corpus")],
                         capture_output=True, text=True, timeout=240)
    assert out.returncode == 0, (out.stdout + out.stderr)[-3000:]
    assert "adapter ok" in out.stdout
