"""The Python host mirror's code tables equal the C ABI's enums in
include/apgar_b200.h (parsed from the header text)."""

import os
import re

import apgar_b200
from apgar_b200 import corridor, dropin

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include",
                      "apgar_b200.h")


def _enum(prefix):
    with open(HEADER) as f:
        text = f.read()
    return {name[len(prefix):].lower(): int(value)
            for name, value in re.findall(r"\b(" + prefix + r"[A-Z0-9_]+)\s*=\s*(\d+)", text)}


def test_path_codes():
    codes = _enum("APGAR_B200_PATH_")
    for value, name in dropin.PATH_CODES.items():
        assert codes[name] == value, name
    for value, name in apgar_b200.LATTICE_PATH_CODES.items():
        assert codes[name] == value, name


def test_predecessor_and_disconnect_codes():
    pred = _enum("APGAR_B200_PRED_")
    assert {v: k for k, v in pred.items()} == dropin.PRED_CODES
    disc = _enum("APGAR_B200_DISCONNECT_")
    assert {v: k for k, v in disc.items()} == dropin.DISCONNECT_CODES


def test_completion_and_corridor_codes():
    comp = _enum("APGAR_B200_COMPLETION_")
    assert comp["reached"] == apgar_b200.COMPLETION_REACHED == 0
    assert comp["disconnected"] == apgar_b200.COMPLETION_DISCONNECTED
    cor = _enum("APGAR_B200_CORRIDOR_")
    assert (cor["none"], cor["certified"], cor["fallback_exit"], cor["fallback_unreached"]) == (
        corridor.NONE, corridor.CERTIFIED, corridor.FALLBACK_EXIT, corridor.FALLBACK_UNREACHED)


def test_generator_codes():
    gen = _enum("APGAR_B200_GENERATOR_")
    assert gen == {"bucketed_frontier": dropin.GENERATOR_FRONTIER,
                   "heading_sweep": dropin.GENERATOR_SWEEP,
                   "b200_persistent": dropin.GENERATOR_PERSISTENT,
                   "b200_persistent_workspace": dropin.GENERATOR_PERSISTENT_WORKSPACE}
