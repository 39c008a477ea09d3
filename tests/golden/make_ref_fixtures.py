"""Writes the reference-mode fixtures under tests/golden/ from the reference's own scene files.

    SR_REFERENCE_DIR=<the reference checkout> python tests/golden/make_ref_fixtures.py

thin_cell.npz: scenes/thin_cell.bin of the reference (crates/sr-engine/tests/gpu/sod.rs:19-24, 560-700: 64 x 64 cells
of the Massive life's step 3,326 — a dense cell (Σ 7.25) between a thin one (Σ 8.4e-4) and denser gas, beside a held
core), its 14 planes as stored (f32) and the life's hold mask.

heat_ceiling.npz, heat_overflow.npz: scenes/heat_ceiling.bin and heat_overflow.bin (crates/sr-engine/tests/gpu/
heat.rs:1413-1431: P5's start in steps 2,517 and 16,127 of two lives, 64 x 64 cells about a thin hot cell beside
vacuum), their 14 planes and the step's Δt (the header's resume.dt_next).

The GPU tests step the reference's own cuts from these files without reading the reference's tree at run time.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from sandbox_reactions_b200 import dump  # noqa: E402


def main():
    ref = os.environ.get("SR_REFERENCE_DIR")
    if not ref:
        sys.exit("set SR_REFERENCE_DIR to the reference checkout")
    d = dump.read(os.path.join(ref, "scenes", "thin_cell.bin"))
    held = d.held if d.held is not None else np.zeros((d.height, d.width), np.uint8)
    out = os.path.join(HERE, "thin_cell.npz")
    np.savez_compressed(out, planes=np.ascontiguousarray(d.planes, np.float32), held=held.astype(np.uint8),
                        dt_next=np.float64(d.dt_next), step=np.int64(d.step))
    print(out, os.path.getsize(out), "bytes")
    for name in ("heat_ceiling", "heat_overflow"):
        d = dump.read(os.path.join(ref, "scenes", name + ".bin"))
        out = os.path.join(HERE, name + ".npz")
        np.savez_compressed(out, planes=np.ascontiguousarray(d.planes, np.float32), dt_next=np.float64(d.dt_next),
                            step=np.int64(d.step))
        print(out, os.path.getsize(out), "bytes")


if __name__ == "__main__":
    main()
