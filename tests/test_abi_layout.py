"""The ctypes mirrors of the C-ABI structs (sdfo/_native.py) against
include/sdfo.h: a C program generated from the ctypes field lists is compiled
with the host compiler and prints each struct's size and each field's
offset, which must equal ctypes' own.  A renamed or missing field fails to
compile; a reordered, retyped or added one changes an offset or a size."""
import ctypes
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# ctypes mirror -> C type
PAIRS = {
    "GridInfo": "sdfo_grid_info",
    "BuildParams": "sdfo_build_params",
    "SparseBuildParams": "sdfo_sparse_build_params",
    "ContactAwareParams": "sdfo_contact_aware_params",
    "MeshDesc": "sdfo_mesh_desc",
    "Pose": "sdfo_pose",
    "BodyState": "sdfo_body_state",
    "ContactParams": "sdfo_contact_params",
    "BEParams": "sdfo_be_params",
    "RigidBody": "sdfo_rigid_body",
    "BuildStats": "sdfo_build_stats",
    "TraversalStats": "sdfo_traversal_stats",
    "Tuning": "sdfo_tuning",
    "DeviceViews": "sdfo_device_views",
}


def test_ctypes_structs_match_header(tmp_path):
    from sdfo import _native as N

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no host C compiler")
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "sdfo.h"', "int main(void) {"]
    expect = []
    for py, c in PAIRS.items():
        cls = getattr(N, py)
        lines.append(f'printf("%zu\\n", sizeof({c}));')
        expect.append(ctypes.sizeof(cls))
        for name, _ in cls._fields_:
            lines.append(f'printf("%zu\\n", offsetof({c}, {name}));')
            expect.append(getattr(cls, name).offset)
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True, capture_output=True)
    got = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True,
                                          text=True).stdout.split()]
    assert got == expect


def test_raw_record_layouts_match_header(tmp_path):
    """Records Python reads as raw tensors: sdfo_be_scene as 26 float64
    (sdfo/be.py: four int32 in the last two slots) and sdfo_contact_measure
    as 5 float64 (sdfo/contact.py: three doubles, then int32 at bytes 24, 28
    and 32)."""
    from sdfo import be

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no host C compiler")
    src = tmp_path / "records.c"
    src.write_text("\n".join([
        "#include <stddef.h>", "#include <stdio.h>", '#include "sdfo.h"', "int main(void) {",
        'printf("%zu %zu %zu\\n", sizeof(sdfo_be_scene), offsetof(sdfo_be_scene, phase), '
        "offsetof(sdfo_be_scene, min_dt_hits));",
        'printf("%zu %zu %zu %zu %zu\\n", sizeof(sdfo_contact_measure), '
        "offsetof(sdfo_contact_measure, normal_velocity), offsetof(sdfo_contact_measure, min_point_index), "
        "offsetof(sdfo_contact_measure, active_count), offsetof(sdfo_contact_measure, valid_count));",
        "return 0;", "}"]) + "\n")
    exe = tmp_path / "records"
    subprocess.run([cc, "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True, capture_output=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    assert [int(x) for x in out[:3]] == [8 * be.SCENE_DOUBLES, 8 * 24, 8 * 24 + 12]
    assert [int(x) for x in out[3:]] == [40, 16, 24, 28, 32]
