"""Generates tests/golden/*.npz from the reference library (run where the reference tree and
oracle/_ref exist; the fixtures are committed, this script is not run by the tests).

    python tests/golden/make_golden.py --reference <reference checkout>

Fixtures (each stores inputs `x` and the reference library's outputs `y0`, `y1`, `y2` for
FORWARD, INVERSE, ROUNDTRIP, computed by oracle/_ref/libbridct_ref.so, i.e. the reference's
own C code built from its sources):

* corpus_<n>.npz   - arrays of the reference's verification corpus dataset/inputs.npz
                     (dataset/corpus.py), each checked against the SHA-256 listed in
                     dataset/manifest.json before use; all cases for n <= 32, a subset above.
                     Also `ids` and `domain` (core / subnormal_diagnostic / range_diagnostic).
* verify_<h>x<w>.npz - the six input families of the reference's tests/verify_plan.py:21-28
                     (zero, impulse at (h//3, w//2), N(0,1) with seed 202609201, ULP
                     neighbours 1 +- 2^-23 in a checkerboard, x 2^-70, x 2^50), for every
                     shape with h, w <= 64.
* configs.npz      - small seeded samples shaped like the benchmark configurations:
                     4 arrays 64x64 U[-1,1] (seed 0), 64 8x8 blocks of a U{0..255}-128 image
                     (seed 1), one 64x128 N(0,1) + smooth term (seed 2), 256x256 log-uniform
                     magnitudes 1e-6..1e6 (seed 4).
"""
from __future__ import annotations

import argparse
import os
import hashlib
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))
from oracle import oracle as O  # noqa: E402

SUBSET = {8: None, 16: None, 32: None, 64: 12, 128: 4, 256: 2}


def ref_outputs(x: np.ndarray):
    return {f"y{m}": O.ref_apply(x, m) for m in range(3)}


def corpus(ref: Path) -> None:
    manifest = json.loads((ref / "dataset" / "manifest.json").read_text())
    with np.load(ref / "dataset" / "inputs.npz", allow_pickle=False) as arrays:
        for n, limit in SUBSET.items():
            cases = [c for c in manifest["cases"] if c["N"] == n]
            if limit is not None:
                # keep the structured cases (cheap to store) and a few random ones
                keep = [c for c in cases if "random" not in c["family"] and "dynamic" not in c["family"]]
                keep = keep[: max(0, limit - 1)] + [c for c in cases if c not in keep][:1]
                cases = keep
            xs, ids, dom = [], [], []
            for c in cases:
                x = arrays[c["id"]]
                digest = hashlib.sha256(x.astype("<f4").tobytes(order="C")).hexdigest()
                if digest != c["sha256"]:
                    raise SystemExit(f"corpus array {c['id']} does not match its manifest digest")
                xs.append(x.astype(np.float32))
                ids.append(c["id"])
                dom.append(c["domain"])
            x = np.stack(xs)
            np.savez_compressed(HERE / f"corpus_{n}.npz", x=x, ids=np.array(ids), domain=np.array(dom),
                                **ref_outputs(x))
            print(f"corpus_{n}: {len(ids)} arrays")


def verify_families(h: int, w: int, rng) -> np.ndarray:
    random = rng.normal(size=(h, w)).astype(np.float32)
    alt = np.where(np.indices((h, w)).sum(axis=0) % 2, 1.0, -1.0).astype(np.float32)
    impulse = np.zeros((h, w), np.float32)
    impulse[h // 3, w // 2] = 1
    return np.stack([np.zeros_like(impulse), impulse, random, (1 + alt * 2 ** -23).astype(np.float32),
                     (random * 2.0 ** -70).astype(np.float32), (random * 2.0 ** 50).astype(np.float32)])


def verify_sets() -> None:
    rng = np.random.default_rng(202609201)
    for h in (8, 16, 32, 64, 128, 256, 512, 1024):
        for w in (8, 16, 32, 64, 128, 256, 512, 1024):
            x = verify_families(h, w, rng)   # advance the generator exactly as the reference does
            if h <= 64 and w <= 64:
                np.savez_compressed(HERE / f"verify_{h}x{w}.npz", x=x, **ref_outputs(x))


def configs() -> None:
    out = {}
    x1 = np.random.default_rng(0).uniform(-1, 1, (1024, 64, 64)).astype(np.float32)[:4]
    out["c1_x"] = x1
    img = (np.random.default_rng(1).integers(0, 256, (4096, 4096)) - 128).astype(np.float32)
    blocks = img[:64, :64].reshape(8, 8, 8, 8).transpose(0, 2, 1, 3).reshape(64, 8, 8).copy()
    out["c2_x"] = blocks
    rng2 = np.random.default_rng(2)
    yy, xx = np.mgrid[0:64, 0:128]
    x3 = (rng2.standard_normal((64, 128)) + np.sin(2 * np.pi * xx / 97) * np.cos(2 * np.pi * yy / 61))
    out["c3_x"] = x3.astype(np.float32)[None]
    rng4 = np.random.default_rng(4)
    mag = 10.0 ** rng4.uniform(-6, 6, (1, 256, 256))
    out["c5_x"] = (mag * rng4.choice([-1.0, 1.0], size=mag.shape)).astype(np.float32)
    for k in list(out):
        ys = ref_outputs(out[k])
        for m in range(3):
            out[k.replace("_x", f"_y{m}")] = ys[f"y{m}"]
    np.savez_compressed(HERE / "configs.npz", **out)


def main() -> None:
    ap = argparse.ArgumentParser()
    env = os.environ.get("BRIDCT_REFERENCE")
    ap.add_argument("--reference", type=Path, default=Path(env) if env else None, required=env is None,
                    help="the reference checkout (default: $BRIDCT_REFERENCE)")
    args = ap.parse_args()
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libbridct_ref.so is missing: run `make -C oracle ref` first")
    corpus(args.reference)
    verify_sets()
    configs()


if __name__ == "__main__":
    main()
