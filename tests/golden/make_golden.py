"""Generates tests/golden/golden.npz: the oracle's outputs (the reference's own World::step, built by
oracle/Makefile) on seeded scenes. The GPU parity tests compare against these vectors when the oracle
library is not at hand, and test_oracle_pins checks the oracle still reproduces them.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)

import reference as R  # noqa: E402
from parity import contact_table  # noqa: E402
from twofold_b200 import scenes  # noqa: E402


def _record(worlds, settings, dt, steps, with_contacts):
    refs = [R.RefWorld(w, settings) for w in worlds]
    for r in refs:
        r.step(dt, steps)
    out = {}
    st = [r.states() for r in refs]
    for k in ("p", "q", "v", "w"):
        out[k] = np.concatenate([s[k] for s in st])
    out["awake"] = np.concatenate([s["awake"] for s in st]).astype(np.int32)
    if with_contacts:
        cands = [r.candidates() for r in refs]
        out["candidates"] = np.concatenate(cands).astype(np.uint64)
        out["candidate_counts"] = np.array([len(c) for c in cands], np.int64)
        exact, pts = [], []
        for r in refs:
            e, p = contact_table(r.contacts(mode=1))
            exact.extend(e)
            pts.append(p)
        out["contacts_exact"] = np.array(exact, np.int64).reshape(-1, 6)
        out["contacts_points"] = np.concatenate(pts).astype(np.float32).reshape(-1, 8)
    return out


def scene_of(name):
    if name == "pyramid":
        sc = scenes.config1()
        return sc.worlds, sc.settings, sc.dt
    if name == "boxes12":
        sc = scenes.Scene("boxes12", [scenes.single("boxes", n=12, seed=3)])
        return sc.worlds, sc.settings, sc.dt
    if name == "uneven4":
        sc = scenes.config4(n_worlds=4)
        return sc.worlds, sc.settings, sc.dt
    if name == "impact2":
        sc = scenes.config5(n_worlds=2)
        return sc.worlds, sc.settings, sc.dt
    raise ValueError(name)


# name -> (scene, steps, record contacts)
SPECS = {
    "pyramid_s1": ("pyramid", 1, True),
    "pyramid_s20": ("pyramid", 20, True),
    "boxes12_s60": ("boxes12", 60, True),
    "uneven4_s30": ("uneven4", 30, True),
    "impact2_s30": ("impact2", 30, True),
}


def _case(name):
    scene, steps, contacts = SPECS[name]

    def run():
        worlds, settings, dt = scene_of(scene)
        return _record(worlds, settings, dt, steps, contacts)

    return run


CASES = {name: _case(name) for name in SPECS}


def main():
    data = {}
    for name, run in CASES.items():
        for k, v in run().items():
            data[f"{name}/{k}"] = v
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **data)
    print("wrote", os.path.join(HERE, "golden.npz"), sum(v.nbytes for v in data.values()), "bytes raw")


if __name__ == "__main__":
    main()
