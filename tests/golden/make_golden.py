"""Generate the golden fixtures that pin the oracle to the reference.

The reference checks in no golden vectors (its bench logs refer to ECG/metal
files that are missing).  This script runs the reference's own UCR Suite
search binaries -- compiled from the reference sources by ``make -C oracle
ref`` -- on small seeded synthetic inputs, and records their outputs next to
the inputs:

    <case>.stream.npy   float32 stream
    <case>.query.npy    float32 query
    golden.json         per case: tool, M, band argument, UCR location/distance

Run from the repository root where the reference tree is present:

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from cudadtw_b200 import synth  # noqa: E402

# (name, generator, N, M, band spec, query seed, noise)
# band spec: ("P", percent) -> UCR R = percent/100 and W = (int)(M*P*0.01);
#            ("W", w)       -> UCR R = w (absolute, R > 1 branch).
CASES = [
    ("ecg_m128_p10", "ecg", 16384, 128, ("P", 10), 11, 0.05),
    ("ecg_m128_w13", "ecg", 16384, 128, ("W", 13), 11, 0.05),
    ("ecg_m64_p5", "ecg", 12000, 64, ("P", 5), 12, 0.05),
    ("metal_m128_p20", "metal", 32768, 128, ("P", 20), 13, 0.1),
    ("metal_m256_p10", "metal", 32768, 256, ("P", 10), 14, 0.1),
    ("metal_m512_p5", "metal", 40000, 512, ("P", 5), 15, 0.1),
    ("walk_m96_p10", "walk", 9000, 96, ("P", 10), 16, 0.5),
]
ED_CASES = [
    ("ed_ecg_m128", "ecg", 16384, 128, 21, 0.05),
    ("ed_metal_m256", "metal", 20000, 256, 22, 0.1),
]


def make_stream(kind: str, n: int) -> np.ndarray:
    if kind == "ecg":
        return synth.ecg_like(n, seed=100 + n % 97)
    if kind == "metal":
        return synth.metal_like(n, seed=200 + n % 89)
    return synth.random_walk(n, seed=300 + n % 83)


def main() -> None:
    oracle.build()
    meta = {"cases": [], "ed_cases": []}
    for name, kind, n, m, (bk, bv), qseed, noise in CASES:
        x = make_stream(kind, n)
        q, off = synth.cut_query(x, m, seed=qseed, noise=noise)
        r_arg = f"{bv / 100.0:.2f}" if bk == "P" else str(bv)
        w = synth.band_from_percent(m, bv) if bk == "P" else bv
        loc, dist, _, _ = oracle.ucr_dtw(x, q, r_arg)
        np.save(os.path.join(HERE, f"{name}.stream.npy"), x)
        np.save(os.path.join(HERE, f"{name}.query.npy"), q)
        meta["cases"].append({"name": name, "M": m, "W": w, "band": [bk, bv],
                              "ucr_R": r_arg, "cut_offset": off,
                              "ucr_location": loc, "ucr_distance": dist})
        print(name, "W", w, "UCR", loc, dist, "cut", off)
    for name, kind, n, m, qseed, noise in ED_CASES:
        x = make_stream(kind, n)
        q, off = synth.cut_query(x, m, seed=qseed, noise=noise)
        loc, dist, _, _ = oracle.ucr_ed(x, q)
        np.save(os.path.join(HERE, f"{name}.stream.npy"), x)
        np.save(os.path.join(HERE, f"{name}.query.npy"), q)
        meta["ed_cases"].append({"name": name, "M": m, "cut_offset": off,
                                 "ucr_location": loc, "ucr_distance": dist})
        print(name, "UCR_ED", loc, dist, "cut", off)
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(meta, f, indent=1)


if __name__ == "__main__":
    main()
