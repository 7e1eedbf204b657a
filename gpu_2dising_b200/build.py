"""In-tree build of the gasp-b200 native code (sm_100a) and of the test oracle.

``build()`` runs ``make`` in the package directory (libgasp_b200.so and the
``gasp`` CLI) and in ``oracle/`` (the CPU restatement, and -- when the
reference sources are present on this machine -- the reference's own code
compiled into ``oracle/_ref/`` as the test oracle).
"""
from __future__ import annotations

import os
import subprocess

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(PKG_DIR)
# The reference checkout (read only): GASP_REFERENCE_SRC, else a "reference"
# directory beside the repository.
REFERENCE_SRC = os.path.abspath(
    os.environ.get("GASP_REFERENCE_SRC", os.path.join(REPO, os.pardir, "reference")))


def _make(directory, *targets):
    jobs = str(max(1, min(8, os.cpu_count() or 1)))
    subprocess.run(["make", "-j", jobs, "-C", directory, *targets], check=True)


def build(with_oracle=True, with_reference=True):
    _make(PKG_DIR)
    if with_oracle:
        _make(os.path.join(REPO, "oracle"))
        if with_reference and os.path.isdir(os.path.join(REFERENCE_SRC, "src")):
            _make(os.path.join(REPO, "oracle"), f"REF={REFERENCE_SRC}", "ref")


if __name__ == "__main__":
    build()
