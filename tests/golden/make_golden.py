"""Generate the golden fixtures in tests/golden/ from the reference renderer itself.

For each case below, a synthetic BHAC snapshot is written by phx_gen_snapshot (seeded, so the bytes are
reproducible; their SHA-256 is recorded), a config.toml is written with the case's keys, and the reference's own CPU
path -- its headers compiled by oracle/build_ref.py into oracle/_ref/ref_render_fp64 and ref_render_fp32 -- renders
the image.  The per-pixel FreqOut records, per-pixel (steps, nplasma, bad) and the total flux are stored in
<case>.npz, the case description and hashes in golden.json.

Needs the reference tree (oracle/build_ref.py) and the built generator (python -m phoenix_b200.build).
usage: python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from tests.golden.cases import CASES, SNAPSHOTS, write_config  # noqa: E402

GEN = os.path.join(ROOT, "phoenix_b200", "_build", "phx_gen_snapshot")
REF = {p: os.path.join(ROOT, "oracle", "_ref", "ref_render_" + p) for p in ("fp64", "fp32")}


def sha256(path):
    h = hashlib.sha256()
    with open(path, "rb") as f:
        for blk in iter(lambda: f.read(1 << 20), b""):
            h.update(blk)
    return h.hexdigest()


def main():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import build_ref  # noqa: E402
    built = build_ref.build(gpu=False)
    if not built:
        raise SystemExit("reference tree not found")
    meta = {"cases": {}, "snapshots": {}}
    with tempfile.TemporaryDirectory() as tmp:
        for name, snap in SNAPSHOTS.items():
            d = os.path.join(tmp, name)
            os.makedirs(d)
            subprocess.check_call([GEN, "--out", d] + snap["gen_args"], stdout=subprocess.DEVNULL)
            meta["snapshots"][name] = {"gen_args": snap["gen_args"], "sha256": sha256(os.path.join(d, "dump.dat")),
                                       "grid_sha256": sha256(os.path.join(d, "grid.in"))}
        for name, case in CASES.items():
            d = os.path.join(tmp, case["snapshot"])
            cfg = os.path.join(tmp, name + ".toml")
            write_config(cfg, case, os.path.join(d, "dump.dat"), os.path.join(d, "grid.in"), os.path.join(tmp, "out"))
            arrays = {}
            summary = {}
            for prec, exe in REF.items():
                out, st = os.path.join(tmp, name + prec + ".bin"), os.path.join(tmp, name + prec + ".st")
                js = json.loads(subprocess.check_output([exe, cfg, "--out", out, "--stats", st]).decode())
                W, H, F = case["img_width"], case["img_height"], len(case["frequencies"])
                arrays["res_" + prec] = np.fromfile(out).reshape(W, H, F, 6)
                arrays["stats_" + prec] = np.fromfile(st, dtype=np.int64).reshape(W, H, 3)
                summary[prec] = {k: js[k] for k in ("steps", "nplasma", "bad", "flux")}
            np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)
            meta["cases"][name] = {"reference": summary}
            print(name, summary["fp64"]["flux"])
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
