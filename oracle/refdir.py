"""Where the reference source tree is, for the tests that read its fixture files.

Test infrastructure only.  The tree is found through the OLPT_REFERENCE_DIR
environment variable, else through the path the oracle Makefile recorded when it
compiled the reference (oracle/_ref/reference_dir.txt).  None when neither names an
existing directory (the GPU box has no reference tree): callers skip."""
import os

_HERE = os.path.dirname(os.path.abspath(__file__))


def reference_dir():
    cands = [os.environ.get("OLPT_REFERENCE_DIR", "")]
    rec = os.path.join(_HERE, "_ref", "reference_dir.txt")
    if os.path.exists(rec):
        with open(rec) as f:
            cands.append(f.read().strip())
    for c in cands:
        if c and os.path.isdir(os.path.join(c, "src")):
            return c
    return None
