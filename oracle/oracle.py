"""Oracle loader (test infrastructure only: imported by tests/, by
__graft_entry__.smoke() and by bench.py's CPU-baseline leg, never by the
package).

  port()       the C restatement, oracle/librhoracle.so (prefix rho_)
  reference()  RHybrid's own hot-path sources built against oracle/shim,
               oracle/_ref/librhref.so (prefix rhref_); None if not built
  reference_gc()  the same with USE_GRID_CONSTRAINT_COUNTERS compiled in,
               oracle/_ref/librhref_gc.so; None if not built
  reference_corsair()  the same driver with the GPU library's Corsair
               adaptor compiled in, oracle/_ref/librhref_corsair.so
"""
import os
import subprocess

from rhybrid_b200.abi import Library

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_PATH = os.path.join(HERE, "librhoracle.so")
REF_PATH = os.path.join(HERE, "_ref", "librhref.so")
REF_GC_PATH = os.path.join(HERE, "_ref", "librhref_gc.so")
REF_CORSAIR_PATH = os.path.join(HERE, "_ref", "librhref_corsair.so")
GPU_LIB_PATH = os.path.join(HERE, "..", "rhybrid_b200", "librhgpu.so")
# the reference tree: RH_REFERENCE_DIR, else the checkout next to this repository
REF_DIR = os.environ.get("RH_REFERENCE_DIR") or os.path.normpath(os.path.join(HERE, "..", "..", "reference"))

_port = None
_ref = None
_ref_gc = None
_ref_corsair = None


def build(reference: bool = True):
    """Builds the restatement, and the reference library when the reference
    tree is present (it is not on GPU machines, which use the prebuilt file)."""
    subprocess.run(["make", "-s", "-C", HERE, "port"], check=True)
    if reference:
        if os.path.isdir(os.path.join(REF_DIR, "src")):
            subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF_DIR={REF_DIR}"], check=True)
            if os.path.exists(GPU_LIB_PATH):
                subprocess.run(["make", "-s", "-C", HERE, "corsair", f"REF_DIR={REF_DIR}"], check=True)
        elif not os.path.exists(REF_PATH):
            print(f"oracle: no reference tree at {REF_DIR} (set RH_REFERENCE_DIR); the reference build is skipped")


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


def reference_corsair():
    """The reference driver with the Corsair-side adaptor of the GPU library
    compiled in (oracle/_ref/librhref_corsair.so, prefix rhref_, plus
    rhcorsair_run); None if not built."""
    global _ref_corsair
    if _ref_corsair is None:
        if not os.path.exists(REF_CORSAIR_PATH):
            return None
        _ref_corsair = Library(REF_CORSAIR_PATH, "rhref_")
    return _ref_corsair


def corsair_run(ctx, nsteps: int, path: int, device: int = 0):
    """rhcorsair_run on a context of reference_corsair(): nsteps steps through
    the adaptor's plugins and propagate() hook on the GPU, the state brought
    back into the reference's containers."""
    import ctypes as C
    f = ctx.lib.dll.rhcorsair_run
    f.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_char_p, C.c_int32]
    f.restype = C.c_int32
    err = C.create_string_buffer(512)
    if f(ctx.h, nsteps, path, device, err, 512) != 0:
        raise RuntimeError("rhcorsair_run: " + err.value.decode())


def reference_write_data(ctx, params, group_names=()):
    """Runs the reference's own output operator (UserDataOP::writeData,
    src/operator_userdata.cpp:55-312) on a context of a reference library and
    returns the arrays it hands to its VLSV writer, in write order, as
    {name: array}: (N,) for vector size 1, else (N, vector size)."""
    import ctypes as C

    import numpy as np

    lib = ctx.lib
    dll = lib.dll
    f = dll.rhref_write_data
    f.argtypes, f.restype = [C.c_void_p, C.c_char_p, C.c_char_p], C.c_int32
    if f(ctx.h, " ".join(params).encode(), " ".join(group_names).encode()) != 0:
        raise RuntimeError(lib.last_error())
    dll.rhref_data_count.argtypes, dll.rhref_data_count.restype = [C.c_void_p], C.c_int32
    info = dll.rhref_data_info
    info.argtypes = [C.c_void_p, C.c_int32, C.c_char_p, C.c_int32, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    get = dll.rhref_data_get
    get.argtypes = [C.c_void_p, C.c_int32, C.POINTER(C.c_double)]
    out = {}
    for i in range(dll.rhref_data_count(ctx.h)):
        name = C.create_string_buffer(256)
        n, v = C.c_int64(), C.c_int64()
        if info(ctx.h, i, name, 256, C.byref(n), C.byref(v)) != 0:
            raise RuntimeError(lib.last_error())
        a = np.empty(n.value * v.value, dtype=np.float64)
        if get(ctx.h, i, a.ctypes.data_as(C.POINTER(C.c_double))) != 0:
            raise RuntimeError(lib.last_error())
        out[name.value.decode()] = a if v.value == 1 else a.reshape(n.value, v.value)
    return out
