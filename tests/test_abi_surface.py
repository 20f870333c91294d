"""The drop-in boundary without a GPU: libsundog.so loads, exports every
entry point include/sundog_api.h declares, and its struct layouts match the
ctypes mirrors byte for byte (checked by compiling the header with gcc).
When sundog's sources are mounted, its own unchanged scene library
(scenes/scenelib.py) replays every committed scene file against this
library (all calls except the GPU render).
"""

import ctypes
import glob
import os
import re
import subprocess
import sys
import textwrap

import pytest

from sundog_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "sundog_api.h")


def declared_symbols():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"SUNDOG_API[^;(]*?\b(sundog_\w+)\s*\(", src, re.S)))


def test_header_declares_drop_in_and_additive():
    names = declared_symbols()
    assert len(abi.DROP_IN_SYMBOLS) == 27
    for n in abi.DROP_IN_SYMBOLS + abi.ADDITIVE_SYMBOLS:
        assert n in names, n


def test_library_exports_every_declared_symbol(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", abi.LIB_PATH], stdout=subprocess.PIPE,
                         text=True, check=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if l.strip()}
    missing = [n for n in declared_symbols() if n not in exported]
    assert not missing, missing
    for n in declared_symbols():
        assert getattr(lib, n) is not None


def test_struct_layouts_match_ctypes(tmp_path):
    probe = textwrap.dedent("""
        #include <stddef.h>
        #include <stdio.h>
        #include "sundog_api.h"
        #define S(t) printf(#t " %zu\\n", sizeof(t));
        #define O(t, f) printf(#t "." #f " %zu\\n", offsetof(t, f));
        int main(void) {
          S(sundog_xform_step) O(sundog_xform_step, a)
          S(sundog_physics_body) O(sundog_physics_body, velocity) O(sundog_physics_body, thickness)
          S(sundog_device_info) O(sundog_device_info, total_mem_mb) O(sundog_device_info, rtcore_version)
          S(sundog_render_options) O(sundog_render_options, spp) O(sundog_render_options, seed)
          O(sundog_render_options, clamp) O(sundog_render_options, quiet)
          S(sundog_render_ext) S(sundog_render_result) S(sundog_session_stats) S(sundog_trace_counts)
          return 0;
        }
    """)
    c = tmp_path / "probe.c"
    c.write_text(probe)
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-I" + os.path.dirname(HEADER), str(c), "-o", str(exe)], check=True)
    vals = dict(l.split() for l in subprocess.run([str(exe)], stdout=subprocess.PIPE, text=True,
                                                  check=True).stdout.splitlines())
    vals = {k: int(v) for k, v in vals.items()}
    assert vals["sundog_xform_step"] == ctypes.sizeof(abi.XformStep) == 32
    assert vals["sundog_xform_step.a"] == abi.XformStep.a.offset
    assert vals["sundog_physics_body"] == ctypes.sizeof(abi.PhysicsBody)
    assert vals["sundog_physics_body.velocity"] == abi.PhysicsBody.velocity.offset
    assert vals["sundog_physics_body.thickness"] == abi.PhysicsBody.thickness.offset
    assert vals["sundog_device_info"] == ctypes.sizeof(abi.DeviceInfo)
    assert vals["sundog_device_info.total_mem_mb"] == abi.DeviceInfo.total_mem_mb.offset
    assert vals["sundog_device_info.rtcore_version"] == abi.DeviceInfo.rtcore_version.offset
    assert vals["sundog_render_options"] == ctypes.sizeof(abi.RenderOptions)
    for f in ("spp", "seed", "clamp", "quiet"):
        assert vals["sundog_render_options." + f] == getattr(abi.RenderOptions, f).offset
    assert vals["sundog_render_ext"] == ctypes.sizeof(abi.RenderExt)
    assert vals["sundog_render_result"] == ctypes.sizeof(abi.RenderResult)
    assert vals["sundog_session_stats"] == ctypes.sizeof(abi.SessionStats)
    assert vals["sundog_trace_counts"] == ctypes.sizeof(abi.TraceCounts)


def test_last_error_is_per_thread(lib):
    import threading
    h = lib.sundog_scene_create(None)
    assert lib.sundog_add_material_lambert(h, None, 7) == -1
    main_msg = abi.last_error(lib)
    seen = {}

    def other():
        seen["msg"] = lib.sundog_last_error()

    t = threading.Thread(target=other)
    t.start()
    t.join()
    assert "texture id out of range" in main_msg
    assert seen["msg"] == b""
    lib.sundog_scene_destroy(h)


from oracle.refpath import reference_root

REF_SCENES = os.path.join(reference_root() or "", "scenes")


@pytest.mark.skipif(not os.path.isdir(REF_SCENES), reason="reference sources not mounted")
def test_reference_scene_files_replay_through_unchanged_scenelib(lib, tmp_path):
    """Every scenes/*.py program, flattened by the reference's own scenelib
    and replayed by its own ctypes layer (_apply) against this library."""
    script = textwrap.dedent("""
        import glob, os, sys, json
        sys.path.insert(0, %(scenes)r)
        os.environ["SUNDOG_BUILD"] = %(build)r
        import scenelib
        lib = scenelib._load_backend()
        done = {}
        for f in sorted(glob.glob(os.path.join(%(scenes)r, "*.py"))):
            if f.endswith("scenelib.py"):
                continue
            g = {"__name__": "replay", "__file__": f}
            sys.argv = [f]
            exec(compile(open(f).read(), f, "exec"), g)
            s = g["s"]
            s.validate()
            h = scenelib._apply(lib, s._program(os.path.dirname(f)))
            assert lib.sundog_scene_validate(h) == 0
            lib.sundog_scene_destroy(h)
            done[os.path.basename(f)] = len(s._objects)
        print(json.dumps(done))
    """) % {"scenes": REF_SCENES, "build": os.path.dirname(abi.LIB_PATH)}
    p = tmp_path / "replay.py"
    p.write_text(script)
    r = subprocess.run([sys.executable, str(p)], stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    import json
    done = json.loads(r.stdout.strip().splitlines()[-1])
    assert len(done) == 19
    # object counts as in the reference's benchmark table (docs/BENCHMARKS.md:9-25)
    assert done["05-spot-swarm.py"] == 32770
    assert done["14-toy-factory.py"] == 55
    assert done["06-spot-cascade.py"] == 518
