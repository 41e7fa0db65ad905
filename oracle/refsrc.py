"""Where the reference checkout lies (TEST INFRASTRUCTURE ONLY).

The reference's sources and input files are read in place, never copied: by
oracle/Makefile.ref (which builds oracle/_ref from them), the fixture generators under
tests/golden/ and the tests that open the reference's own geometry and parameter files.
CSP_REFERENCE_DIR names the checkout; unset, the recipe's default location is used.
reference_file() returns None when the file is absent (tests then skip), so nothing on a
machine without the checkout reads it.
"""
import os

DEFAULT = "/root/reference"


def reference_dir():
    """The reference checkout, or None when it is not on this machine."""
    d = os.environ.get("CSP_REFERENCE_DIR") or DEFAULT
    return d if os.path.isdir(d) else None


def reference_file(*parts):
    """Path of a file of the reference checkout, or None when it is absent."""
    d = reference_dir()
    if d is None:
        return None
    p = os.path.join(d, *parts)
    return p if os.path.exists(p) else None
