#!/usr/bin/env python3
"""Where the reference checkout lies, for the oracle's build recipe.

TEST INFRASTRUCTURE ONLY.  $CT_REF_DIR when set, else the `reference_path`
the workload description (BASELINE.json at the repository root) records.
Prints the path; prints nothing when neither names one."""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def reference_dir():
    d = os.environ.get("CT_REF_DIR")
    if d:
        return d
    try:
        with open(os.path.join(os.path.dirname(HERE), "BASELINE.json")) as f:
            return json.load(f).get("reference_path") or ""
    except (OSError, ValueError):
        return ""


if __name__ == "__main__":
    sys.stdout.write(reference_dir())
