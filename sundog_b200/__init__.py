"""sundog_b200 — a B200-native (sm_100a) path tracer behind sundog's C ABI.

libsundog.so (built in-tree from csrc/ by build.py) exports the reference
renderer's 27-symbol scene/render ABI plus additive entry points; abi.py
binds it with ctypes, scene.py mirrors the reference scene library's builder
API, workloads.py generates the seeded benchmark scenes.
"""

__all__ = ["abi", "scene", "workloads", "build"]
