"""Regenerate the ball fixture from the reference tree.

The reference ships an analytic cone-beam simulation of a ball
(``Tomography_3D/Simul_Data``: ``boule.obj`` phantom, ``boule.data`` its
16^3 voxel image, ``proj_boule.data`` 720 projections of 32 x 32 cells, both
float32 after a 512-byte header, made by ``simu.sh``).  This script copies
the phantom file and the image verbatim and keeps every 45th projection
(16 views, header record count updated) so the fixture stays small:

    python tests/golden/make_ball.py [reference_root]

(reference_root defaults to $TRTT_REFERENCE_ROOT, else /root/reference).

Outputs: tests/golden/ball/{boule.obj, boule.data, proj_boule_every45.data}.
"""
import os
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
EVERY = 45


def main(root=None):
    root = root or os.environ.get("TRTT_REFERENCE_ROOT", "/root/reference")
    src = os.path.join(root, "Tomography_3D", "Simul_Data")
    dst = os.path.join(HERE, "ball")
    os.makedirs(dst, exist_ok=True)
    shutil.copyfile(os.path.join(src, "boule.obj"), os.path.join(dst, "boule.obj"))
    shutil.copyfile(os.path.join(src, "boule.data"), os.path.join(dst, "boule.data"))
    raw = np.fromfile(os.path.join(src, "proj_boule.data"), dtype="<f4")
    header, data = raw[:128].copy(), raw[128:].reshape(720, 32, 32)
    keep = data[::EVERY]
    header[3] = keep.shape[0]
    with open(os.path.join(dst, f"proj_boule_every{EVERY}.data"), "wb") as f:
        f.write(header.tobytes())
        f.write(np.ascontiguousarray(keep).tobytes())


if __name__ == "__main__":
    main(*sys.argv[1:])
