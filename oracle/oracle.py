"""Oracle loader (test infrastructure only: imported by tests/, by
__graft_entry__.smoke() and by bench.py's CPU-baseline leg, never by the
package).

  port()       the C restatement, oracle/librhoracle.so (prefix rho_)
  reference()  RHybrid's own hot-path sources built against oracle/shim,
               oracle/_ref/librhref.so (prefix rhref_); None if not built
  reference_gc()  the same with USE_GRID_CONSTRAINT_COUNTERS compiled in,
               oracle/_ref/librhref_gc.so; None if not built
"""
import os
import subprocess

from rhybrid_b200.abi import Library

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_PATH = os.path.join(HERE, "librhoracle.so")
REF_PATH = os.path.join(HERE, "_ref", "librhref.so")
REF_GC_PATH = os.path.join(HERE, "_ref", "librhref_gc.so")
REF_DIR = os.environ.get("RH_REFERENCE_DIR", "/root/reference")

_port = None
_ref = None
_ref_gc = None


def build(reference: bool = True):
    """Builds the restatement, and the reference library when the reference
    tree is present (it is not on GPU machines, which use the prebuilt file)."""
    subprocess.run(["make", "-s", "-C", HERE, "port"], check=True)
    if reference and os.path.isdir(os.path.join(REF_DIR, "src")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF_DIR={REF_DIR}"], check=True)


def port() -> Library:
    global _port
    if _port is None:
        if not os.path.exists(PORT_PATH):
            build(reference=False)
        _port = Library(PORT_PATH, "rho_")
    return _port


def reference():
    global _ref
    if _ref is None:
        if not os.path.exists(REF_PATH):
            return None
        _ref = Library(REF_PATH, "rhref_")
    return _ref


def reference_gc():
    global _ref_gc
    if _ref_gc is None:
        if not os.path.exists(REF_GC_PATH):
            return None
        _ref_gc = Library(REF_GC_PATH, "rhref_")
    return _ref_gc
