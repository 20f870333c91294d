"""Generates the reference-image fixtures (run where sundog's sources are
mounted; the GPU box does not need them):

  ref_<scene>.png    sundog's own golden render of the scene (tests/golden/
                     <scene>.avif: 256x256, 64 spp, seed 7, no denoise, 12-bit
                     PQ BT.2020 lossless AVIF from its OptiX build), decoded
                     by Pillow to 8 bits per channel and stored losslessly;
  abi_<scene>.json   the C-ABI call stream sundog's unchanged scene library
                     (scenes/scenelib.py `_apply`) sends for the scene file:
                     every call with its arguments as plain values and its
                     return code, recorded through a forwarding proxy in front
                     of this repository's libsundog.so as scenelib loads it
                     (scene building only, no GPU).

Scenes: the goldens that need no asset files (smoke, 01-marble-run,
02-cornell-lume); the others load AVIF textures, OBJ meshes or an HDRI from
sundog's asset tree.

Usage: python tests/golden/make_reference_images.py [sundog-root]
"""
import ctypes
import json
import os
import sys

import numpy as np
from PIL import Image

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from sundog_b200 import abi  # noqa: E402  (library path)

SCENES = ["smoke", "01-marble-run", "02-cornell-lume"]


def encode(a):
    """A ctypes call argument as a JSON value (decoded by the replay in
    tests/test_gpu_reference_images.py)."""
    if a is None or isinstance(a, (bool, int, float)):
        return a
    if isinstance(a, bytes):
        return {"s": a.decode()}
    if isinstance(a, ctypes.c_void_p):
        return {"h": 0}
    if isinstance(a, (ctypes.c_double, ctypes.c_float, ctypes.c_int, ctypes.c_int64)):
        return a.value
    if isinstance(a, ctypes.Array):
        if a._type_ is ctypes.c_double:
            return {"d": list(a)}
        if issubclass(a._type_, ctypes.Structure):  # transform steps
            return {"xf": [fields(x) for x in a]}
    obj = getattr(a, "_obj", None)  # ctypes.byref(struct): the physics block
    if isinstance(obj, ctypes.Structure):
        return {"pb": fields(obj)}
    raise TypeError("unrecorded argument type %r" % type(a))


def fields(st):
    """A ctypes structure as {field: value} (the ABI's field names)."""
    out = {}
    for name, _ in st._fields_:
        v = getattr(st, name)
        out[name] = list(v) if isinstance(v, ctypes.Array) else v
    return out


class Recorder(object):
    def __init__(self, lib):
        self.lib = lib
        self.log = []

    def __getattr__(self, name):
        f = getattr(self.lib, name)
        if not name.startswith("sundog_"):
            return f

        def call(*args):
            entry = [name, [encode(a) for a in args]]
            r = f(*args)
            entry.append(r if isinstance(r, int) else None)
            if name == "sundog_scene_create":
                entry[2] = None
            self.log.append(entry)
            return r
        return call


def main(ref_root):
    scenes_dir = os.path.join(ref_root, "scenes")
    sys.path.insert(0, scenes_dir)
    os.environ["SUNDOG_BUILD"] = os.path.dirname(abi.LIB_PATH)
    import scenelib
    lib = scenelib._load_backend()  # this library, with scenelib's own prototypes
    for name in SCENES:
        img = np.array(Image.open(os.path.join(ref_root, "tests", "golden", name + ".avif")).convert("RGB"))
        Image.fromarray(img).save(os.path.join(HERE, "ref_%s.png" % name), optimize=True)
        f = os.path.join(scenes_dir, name + ".py")
        g = {"__name__": "record", "__file__": f}
        sys.argv = [f]
        exec(compile(open(f).read(), f, "exec"), g)
        s = g["s"]
        s.validate()
        rec = Recorder(lib)
        h = scenelib._apply(rec, s._program(scenes_dir))
        lib.sundog_scene_destroy(h)
        with open(os.path.join(HERE, "abi_%s.json" % name), "w") as out:
            json.dump({"scene": name, "calls": rec.log}, out, separators=(",", ":"))
        print(name, img.shape, len(rec.log), "calls")


if __name__ == "__main__":
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from oracle.refpath import reference_root
    main(sys.argv[1] if len(sys.argv) > 1 else reference_root())
