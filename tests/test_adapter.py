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
PREPARED = os.path.join(ROOT, "apgar_b200", "adapter", "_build", "prepared_batch_check")
PATCH = os.path.join(ROOT, "apgar_b200", "adapter", "reference_generator.patch")


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


def test_generator_patch_applies_to_the_reference(tmp_path):
    """The maintainer's patch (the B200 persistent generators and their
    descriptor) applies cleanly to the reference's own files."""
    import shutil

    import oracle

    ref = oracle.reference_root()
    if ref is None:
        pytest.skip("reference sources are absent (set APGAR_REFERENCE or run oracle/build_ref.sh)")
    for rel in ("include/apgar/gpu/planar_router.h", "src/gpu/planar_router.cc",
                "src/candidates/gpu_candidate_adapter.cc"):
        (tmp_path / rel).parent.mkdir(parents=True, exist_ok=True)
        shutil.copy(os.path.join(ref, rel), tmp_path / rel)
    with open(PATCH) as f:
        out = subprocess.run(["patch", "-p1", "--dry-run"], cwd=tmp_path, stdin=f,
                             capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr


@pytest.mark.gpu
def test_prepared_batch_path_of_the_reference_on_gpu():
    """RouteCandidateBatchWithPreparedPlanarGpuBackend of the patched reference
    over this backend: every corpus item sealed at the CPU A* cost, every
    sealed item turned into a route candidate by the reference's candidate
    adapter and admitted, and every fault class raises the reference's
    invariant id."""
    import re

    if not os.path.exists(PREPARED):
        pytest.skip("prepared-path check not built (needs the reference sources at build time)")
    out = subprocess.run([PREPARED], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, (out.stdout + out.stderr)[-4000:]
    m = re.search(r"prepared ok: (\d+) cases, (\d+) items sealed at the CPU A\* cost, (\d+) route "
                  r"candidates built and admitted", out.stdout)
    assert m is not None, out.stdout[-2000:]
    cases, sealed, admitted = (int(g) for g in m.groups())
    assert cases == 11 and sealed > 0 and admitted == sealed, m.group(0)
