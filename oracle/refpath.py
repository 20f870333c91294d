"""ORACLE — test infrastructure only.

Location of the mounted reference sources, for the recipes that read them in
place (oracle/Makefile `make ref`, the golden-fixture scripts under
tests/golden/) and the tests that replay the reference's own files. The
environment variable SUNDOG_REFERENCE names the reference checkout; without
it the recipes look at the one mount point this project's build machines
use. Nothing here is needed where the reference is absent: the prebuilt
oracle/_ref libraries travel with the repository, and code that needs the
sources checks for None.
"""

import os

_DEFAULT_MOUNT = "/root/reference"


def reference_root():
    """The reference checkout's root directory, or None when it is absent."""
    r = os.environ.get("SUNDOG_REFERENCE")
    if r:
        return r if os.path.isdir(r) else None
    return _DEFAULT_MOUNT if os.path.isdir(_DEFAULT_MOUNT) else None
