"""B200-native XPBD Gaussian-graph solver step behind the reference ``xpbd_*`` C ABI.

The product is the shared library ``libxpbd_b200.so`` built from ``csrc/`` (host C++
and hand-written sm_100a CUDA kernels).  This package only locates and binds it:

* ``XPBD(...)`` — the drop-in ctypes bridge with the reference's method set
  (src/xpbd_bridge.py:45-271), bound to this package's library by default;
* ``library_path()`` — the in-tree library path (the value to put in ``XPBD_DLL``
  for the reference's own bridge);
* ``scenes`` — seeded synthetic workloads;
* ``batch`` — many independent objects packed into one scene;
* ``serve`` — continuous-batching session loop over resident engine instances;
* ``graph_io`` — APGGRPH1 graphs, graph ``.npz`` renumbering, 3DGS PLY, runtime inputs;
* ``splat`` — cameras for the splatting pass (``XPBD.render``).

There is no CPU fallback: constructing ``XPBD`` without the built library raises.
"""
import os

from . import batch, bridge, graph_io, scenes, serve, splat  # noqa: F401

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_NAME = "libxpbd_b200.so"


def library_path():
    return os.path.join(PKG_DIR, LIB_NAME)


def XPBD(dll_path=None, instance=False):
    """The reference bridge's ``XPBD`` bound to the B200 library (or ``dll_path``); with
    ``instance=True`` an engine of its own instead of the library's singleton."""
    path = dll_path or os.environ.get("XPBD_B200_DLL") or library_path()
    if not os.path.isfile(path):
        raise FileNotFoundError(
            f"{path} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'` "
            "or `make -C 3dgs-isaac-sim-xpbd_b200/csrc`")
    return bridge.XPBD(path, instance=instance)
