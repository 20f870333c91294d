"""The numpy FP64 restatement of sundog's sampling-table builds
(oracle/tables.py) against the CPU oracle's C++ build of the same tables
(oracle/integrator.cpp, the reference's loops): bit for bit, for the
instancing workload's 1024x512 sky and the volumes workload's 2048-triangle
canopy light."""

import os

import numpy as np

from oracle import oracle, tables
from sundog_b200 import workloads


def test_env_tables_restatement_matches_oracle(oracle_lib, asset_dir):
    s = workloads.instancing(asset_dir, width=32, height=18, spp=1)
    text, _ = oracle.reference_scene_text(s, asset_dir)
    osc = oracle.OracleScene(text)
    try:
        om, oc = osc.table(0), osc.table(1)
    finally:
        osc.close()
    m, c, m64, c64 = tables.env_tables(tables.read_rgbe(os.path.join(asset_dir,
                                                                     "sky_1024x512.hdr")))
    assert om.tobytes() == m.tobytes()
    assert oc.tobytes() == c.ravel().tobytes()


def test_mesh_light_restatement_matches_oracle(oracle_lib, asset_dir):
    s = workloads.volumes(asset_dir, width=32, height=18, spp=1)
    text, _ = oracle.reference_scene_text(s, asset_dir)
    obj = [l.split() for l in text.split("\n") if l.startswith("object 5")][0]
    light, xf = int(obj[6]), [float(x) for x in obj[7:19]]
    osc = oracle.OracleScene(text)
    try:
        ocdf = osc.table(2 + light)
    finally:
        osc.close()
    pos, tris = tables.read_obj_triangles(os.path.join(asset_dir, "canopy_2048.obj"))
    cdf, cdf64, total = tables.mesh_light_cdf(pos, tris, xf)
    assert len(cdf) == 2049 and total > 0
    assert ocdf.tobytes() == cdf.tobytes()
