"""The ctypes mirrors of the C ABI structs (renderbox2_b200/_native.py,
scenefile.py, serve.py) match the layouts in include/*.h: a C program built
with gcc from the headers prints every struct's size and every mirrored
field's offset, and each must equal ctypes' figure.  A field added to a
header but not to its mirror (or the reverse) shows up as a size or offset
mismatch, or as a compile error naming the field.  CPU only."""
import ctypes as C
import shutil
import subprocess
from pathlib import Path

import pytest

from renderbox2_b200 import _native as N
from renderbox2_b200 import scenefile as SF
from renderbox2_b200 import serve as SV

ROOT = Path(__file__).resolve().parents[1]

MIRRORS = {
    "rb2_build_params": N.BuildParams, "rb2_bvh_counts": N.BvhCounts, "rb2_cw8_counts": N.Cw8Counts,
    "rb2_launch_config": N.LaunchConfig, "rb2_trace_job": N.TraceJob, "rb2_host_job": N.HostJob,
    "rb2_dev_bvh": N.DevBvh, "rb2_dev_scene": N.DevScene, "rb2_isect_buffer": N.IsectBuffer,
    "rb2_bsdf_layer": N.BsdfLayer, "rb2_material_desc": N.MaterialDesc, "rb2_filter": N.Filter,
    "rb2_batch_config": N.BatchConfig, "rb2_ao_params": N.AoParams, "rb2_pt_params": N.PtParams,
    "rb2_bdpt_params": N.BdptParams, "rb2_bdpt_lvc_params": N.BdptLvcParams, "rb2_raycast_params": N.RayCastParams,
    "rb2_render_stats": N.RenderStats, "rb2_camera": N.Camera, "rb2_scene_file_info": SF.SceneFileInfo,
    "rb2_job": SV.Job, "rb2_job_result": SV.JobResult, "rb2_server_config": SV.ServerConfig,
    "rb2_server_stats": SV.ServerStats,
}


def _c_layouts(tmp_path):
    lines = ['#include "rb2.h"', '#include "rb2_render.h"', '#include "rb2_scene.h"', '#include "rb2_serve.h"',
             "#include <stddef.h>", "#include <stdio.h>", "int main(void) {"]
    for cname, cls in MIRRORS.items():
        lines.append(f'  printf("{cname} %zu\\n", sizeof({cname}));')
        for field, _ in cls._fields_:
            lines.append(f'  printf("{cname}.{field} %zu\\n", offsetof({cname}, {field}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layouts.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layouts"
    r = subprocess.run(["gcc", "-std=c11", "-Wall", f"-I{ROOT / 'include'}", str(src), "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    return {k: int(v) for k, v in (ln.split() for ln in out.splitlines())}


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc not found")
def test_ctypes_mirrors_match_the_headers(tmp_path):
    c = _c_layouts(tmp_path)
    bad = []
    for cname, cls in MIRRORS.items():
        if c[cname] != C.sizeof(cls):
            bad.append(f"sizeof({cname}) = {c[cname]}, ctypes {cls.__name__} = {C.sizeof(cls)}")
        for field, _ in cls._fields_:
            off = getattr(cls, field).offset
            if c[f"{cname}.{field}"] != off:
                bad.append(f"offsetof({cname}, {field}) = {c[cname + '.' + field]}, ctypes = {off}")
    assert not bad, "\n".join(bad)
