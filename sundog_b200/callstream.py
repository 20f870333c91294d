"""Recorded C-ABI call streams as scenes.

A call stream is the exact sequence of scene-construction calls a program
sent to libsundog.so, recorded as JSON ({"scene": name, "calls": [[function,
args, return value], ...]}; tests/golden/abi_*.json hold the streams sundog's
own scenelib sends for its golden scenes). CallStreamScene replays one against
any library that exports the scene ABI (this package's libsundog.so, or the
oracle's build of sundog's own scene code), so a recorded scene renders,
benchmarks and derives exactly as the original program would have had it.
Arguments are encoded as: {"h": 0} the scene handle, {"s": text} the base
directory, {"d": [...]} a double array, {"xf": [...]} transform steps,
{"pb": {...}} a physics body; plain JSON values otherwise.
"""

import ctypes
import json

from . import abi


def _decode(a, handle, base_dir):
    if isinstance(a, dict):
        if "h" in a:
            return handle
        if "s" in a:
            return base_dir.encode()
        if "d" in a:
            return (ctypes.c_double * len(a["d"]))(*a["d"])
        if "xf" in a:
            return (abi.XformStep * len(a["xf"]))(*[abi.XformStep(**f) for f in a["xf"]])
        if "pb" in a:
            f = dict(a["pb"])
            for k in ("velocity", "angular_velocity"):
                f[k] = (ctypes.c_double * 3)(*f[k])
            return ctypes.byref(abi.PhysicsBody(**f))
        raise ValueError("call stream: unknown argument encoding %r" % (a,))
    if isinstance(a, str):
        return a.encode()
    return a


def replay(lib, calls, base_dir="."):
    """Rebuilds the scene from a call stream; every call must return what it
    returned when recorded. Returns the scene handle (the caller destroys
    it)."""
    h = None
    try:
        for name, args, ret in calls:
            r = getattr(lib, name)(*[_decode(a, h, base_dir) for a in args])
            if name == "sundog_scene_create":
                if not r:
                    raise abi.SundogError("call stream: " + abi.last_error(lib))
                h = r
            elif r != ret:
                raise abi.SundogError("call stream: %s returned %r, recorded %r (%s)" %
                                      (name, r, ret, abi.last_error(lib)))
    except Exception:
        if h:
            lib.sundog_scene_destroy(h)
        raise
    return h


class CallStreamScene(object):
    """A recorded scene with the builder interface of sundog_b200.scene.Scene
    (build(base_dir, lib) -> handle), so sessions, renders and the oracle take
    it like a scene built in Python."""

    def __init__(self, path):
        with open(path) as f:
            d = json.load(f)
        self.name = d.get("scene", path)
        self.calls = d["calls"]

    def build(self, base_dir=".", lib=None):
        return replay(lib or abi.load(), self.calls, base_dir)
