"""Writes tests/golden/replay_invariants.json: for each of the reference's
GPU replay artifacts (replays/gpu/*.replay, key=value text), the injected
fault, the generator, and the failure and invariant id the reference's host
validation must raise.  Run where the reference tree is present:

    python tests/golden/make_replay_invariants.py [reference root]
"""

import glob
import json
import os
import sys

KEYS = ("generator", "fault", "expected_failure", "expected_invariant")


def main(root: str) -> None:
    rows = []
    for path in sorted(glob.glob(os.path.join(root, "replays", "gpu", "*.replay"))):
        fields = {}
        with open(path) as f:
            for line in f:
                key, sep, value = line.strip().partition("=")
                if sep and key in KEYS:
                    fields[key] = value
        rows.append(dict(replay=os.path.basename(path), **fields))
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "replay_invariants.json")
    with open(out, "w") as f:
        json.dump(rows, f, indent=1)
    print(out, len(rows))


if __name__ == "__main__":
    if len(sys.argv) > 1:
        root = sys.argv[1]
    else:
        sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))
        import oracle

        root = oracle.reference_root()
        if root is None:
            sys.exit("usage: make_replay_invariants.py REFERENCE_ROOT (or set APGAR_REFERENCE)")
    main(root)
