"""Generate the golden vectors committed under tests/golden/.

Two sources:

1. ``reference_fixtures.npz`` -- a subset of AutoRIFT.jl's own OpenCV fixtures
   (test/fixtures/matchtemplate/zncc_*, pyrup/*, peak/*, generated upstream by
   tools/python_ref/gen_fixtures.py with OpenCV 4.10), repacked so the tests can run where the
   reference tree is absent. Read from the reference checkout given by --reference.
2. ``opencv_golden.npz`` -- new seeded cases computed here with the installed OpenCV
   (cv2.matchTemplate TM_CCOEFF_NORMED, cv2.pyrUp), covering geometries the reference fixtures
   do not: non-square chips, independent radii, uint16 windows.

Run:  python tests/golden/make_golden.py --reference /path/to/AutoRIFT.jl
"""

from __future__ import annotations

import argparse
import json
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def load_fixture(root: Path, name: str):
    d = root / "test" / "fixtures" / name
    meta = json.loads((d / "meta.json").read_text())
    arrays = {k: np.fromfile(d / f"{k}.bin", dtype=spec["dtype"]).reshape(spec["shape"])
              for k, spec in meta["arrays"].items()}
    return arrays, meta["params"]


def pack_reference(root: Path) -> dict:
    out = {}
    names = []
    for cs in (32, 64, 128):
        for r in (6, 10, 25):
            for dt, var in (("uint8", "plain"), ("float32", "plain"), ("float32", "dc_offset"),
                            ("float32", "lowcontrast")):
                if cs == 128 and dt == "float32":
                    continue  # the largest float cases stay in the reference tree only
                names.append(f"matchtemplate/zncc_c{cs}_r{r}_{dt}_{var}")
    for patch in ("random", "delta", "plateau", "monotone", "equal"):
        for f in (2, 4, 8):
            names.append(f"pyrup/{patch}_step_x{f}")
            names.append(f"pyrup/{patch}_cascade_x{f}")
    for p in ("unique", "tie_in_row", "tie_in_column", "plateau", "all_equal"):
        names.append(f"peak/{p}")
    meta = {}
    for name in names:
        arrays, params = load_fixture(root, name)
        key = name.replace("/", "__")
        for k, v in arrays.items():
            out[f"{key}::{k}"] = v
        meta[key] = params
    out["__meta__"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    return out


def make_opencv() -> dict:
    import cv2

    out = {}
    meta = {"opencv_version": cv2.__version__, "cases": []}
    rng = np.random.default_rng(20261203)
    cases = [
        ("u8_c32x16_r9x13", np.uint8, (16, 32), (9, 13)),   # (ch, cw), (rx, ry)
        ("u8_c24_r7", np.uint8, (24, 24), (7, 7)),
        ("f32_c40x32_r12x5", np.float32, (32, 40), (12, 5)),
        ("u16_c32_r10", np.uint16, (32, 32), (10, 10)),
    ]
    for name, dt, (ch, cw), (rx, ry) in cases:
        wr, wc = ch + 2 * ry - 1, cw + 2 * rx - 1
        base = rng.standard_normal((wr + 8, wc + 8))
        base = cv2.GaussianBlur(base, (0, 0), 1.2)
        base = (base - base.min()) / (base.max() - base.min())
        if dt == np.uint8:
            search = np.round(base[:wr, :wc] * 255).astype(np.uint8)
        elif dt == np.uint16:
            search = np.round(base[:wr, :wc] * 40000 + 8000).astype(np.uint16)
        else:
            search = (base[:wr, :wc] * 0.4 + 0.3).astype(np.float32)
        # The chip is the window content at a known shift plus a little noise.
        oy, ox = int(rng.integers(0, 2 * ry)), int(rng.integers(0, 2 * rx))
        chip = search[oy:oy + ch, ox:ox + cw].astype(np.float64)
        chip = chip + rng.normal(0, 0.01 * (chip.std() + 1e-9), chip.shape)
        chip = np.clip(np.round(chip), 0, np.iinfo(dt).max).astype(dt) if dt != np.float32 else chip.astype(dt)
        s32 = search.astype(np.float32)
        c32 = chip.astype(np.float32)
        expected = cv2.matchTemplate(s32, c32, cv2.TM_CCOEFF_NORMED)
        out[f"{name}::search"] = search
        out[f"{name}::chip"] = chip
        out[f"{name}::expected"] = expected.astype(np.float32)
        meta["cases"].append({"name": name, "rx": rx, "ry": ry, "shift_rc": [oy, ox]})
    # pyrUp cascades of random 5x5 patches to x16 (160x160), BORDER_REFLECT_101 default.
    for k in range(3):
        p = rng.standard_normal((5, 5)).astype(np.float32)
        cur = p
        for _ in range(4):
            cur = cv2.pyrUp(cur)
        out[f"pyrup_cascade_{k}::src"] = p
        out[f"pyrup_cascade_{k}::expected"] = cur
    out["__meta__"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", type=Path, required=True)
    args = ap.parse_args()
    np.savez_compressed(HERE / "reference_fixtures.npz", **pack_reference(args.reference))
    np.savez_compressed(HERE / "opencv_golden.npz", **make_opencv())
    for f in ("reference_fixtures.npz", "opencv_golden.npz"):
        print(f, (HERE / f).stat().st_size // 1024, "KiB")


if __name__ == "__main__":
    main()
