"""Writes tests/golden/host_setup_digests.json: the host builder's per-array digests
(dpm_setup_host_digest) of the meshes in tests/test_host_setup.py, hex-encoded.  Regenerate only
after a deliberate change of the set-up's arithmetic, and check the new arrays against the device
builder first (tests/test_gpu_setup.py, tests/test_gpu_foam.py).  Run from the repository root:

    python tests/golden/make_host_setup_digests.py
"""
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def main():
    sys.path.insert(0, ROOT)
    from tests.test_host_setup import CASES, GOLDEN, digests_as_hex
    out = {name: digests_as_hex(make()) for name, make in CASES.items()}
    with open(GOLDEN, "w") as fh:
        json.dump(out, fh, indent=1, sort_keys=True)
        fh.write("\n")
    print(f"wrote {GOLDEN}: {len(out)} meshes")


if __name__ == "__main__":
    main()
