"""Copies the reference's shipped scene files that can be rendered here
(no asset listed in its .MISSING_LARGE_BLOBS) into tests/golden/ref_scenes,
with the assets they reference (OBJ meshes, BMP textures), keeping the
paths relative to the reference's root: the reference's parser opens assets
relative to the working directory, and the reference tree is not present
where the GPU tests run. TEST FIXTURES (scene data, not code).

  python tests/golden/make_scene_fixtures.py        [MRT_REFERENCE_DIR=...]
"""
from __future__ import annotations

import os
import re
import shutil
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "ref_scenes"
REF = Path(os.environ.get("MRT_REFERENCE_DIR", "/root/reference"))

# scene files of the reference (scenes/**), and whether all their assets exist
SCENES = ["scenes/subject/sphere.rt", "scenes/subject/cylinder.rt", "scenes/subject/hyper.rt",
          "scenes/subject/detout.rt", "scenes/subject/columns.rt", "scenes/obj/cube.rt"]


def assets_of(rt: Path) -> list[str]:
    out = []
    for line in rt.read_text().splitlines():
        line = line.split("#", 1)[0]
        out += re.findall(r"(assets/\S+)", line)
    return out


def main() -> int:
    if not (REF / "scenes").exists():
        print("reference not found", file=sys.stderr)
        return 1
    for s in SCENES:
        src = REF / s
        missing = [a for a in assets_of(src) if not (REF / a).exists()]
        if missing:
            print(f"skip {s}: missing {missing}")
            continue
        for rel in [s] + assets_of(src):
            dst = OUT / rel
            dst.parent.mkdir(parents=True, exist_ok=True)
            shutil.copyfile(REF / rel, dst)
        print("copied", s)
    return 0


if __name__ == "__main__":
    sys.exit(main())
