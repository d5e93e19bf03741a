"""Copy the reference's committed bundles and golden outputs into tests/golden/.

warp-fdtd commits frozen input bundles (results/warp_reference/<case>/) and the
outputs its own Warp float32 path produced on them (results/warp/<case>/), plus
independent FDTDX outputs (results/<case>/arrays.npz).  The GPU box that runs the
parity tests has no copy of the reference, so this script extracts the subset the
tests need:

* forward50_gpu: bundle (80x80x30, 2098 steps, two flux detectors), Warp full
  3-D E/H after the run (results/warp/forward50_gpu/fields.npz) and the FDTDX
  flux traces (results/forward50_gpu/arrays.npz keys input/output);
* hann_200fs: bundle (200x200x75, 5245 steps, flux + three mode detectors),
  Warp mid-z E/H, Warp mode_in/mode_out phasors (mode_reflected shares
  mode_in's plane, hence its phasors), Warp measurements (result.json), FDTDX
  flux traces;
* gradient20: bundle gradient20_highest_exact, Warp gradient
  (results/warp/gradient20/gradient.npz) and its result.json.

Bundles are copied byte for byte so their manifest SHA-256 still matches.
Run from anywhere:  python tests/golden/make_golden.py /path/to/warp-fdtd
"""

import json
import shutil
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def copy_bundle(ref, case, name):
    dst = HERE / name
    dst.mkdir(parents=True, exist_ok=True)
    for f in ("inputs.npz", "manifest.json"):
        shutil.copyfile(ref / "results" / "warp_reference" / case / f, dst / f)
    return dst


def flux_traces(src, dst):
    with np.load(src) as a:
        keep = {k: a[k] for k in a.files if k not in ("E", "H", "inv_eps")}
    np.savez_compressed(dst, **keep)


def main(ref):
    ref = Path(ref)
    res = ref / "results"

    d = copy_bundle(ref, "forward50_gpu", "forward50_gpu")
    shutil.copyfile(res / "warp/forward50_gpu/fields.npz", d / "warp_fields.npz")
    shutil.copyfile(res / "warp/forward50_gpu/result.json", d / "warp_result.json")
    flux_traces(res / "forward50_gpu/arrays.npz", d / "fdtdx_flux.npz")

    d = copy_bundle(ref, "hann_200fs", "hann_200fs")
    shutil.copyfile(res / "warp/hann20/fields.npz", d / "warp_fields.npz")
    shutil.copyfile(res / "warp/hann20/result.json", d / "warp_result.json")
    for m in ("mode_in", "mode_out"):
        shutil.copyfile(
            res / f"warp/hann20/{m}_phasors.npz", d / f"warp_{m}_phasors.npz"
        )
    flux_traces(res / "hann_200fs/arrays.npz", d / "fdtdx_flux.npz")

    d = copy_bundle(ref, "gradient20_highest_exact", "gradient20")
    shutil.copyfile(res / "warp/gradient20/gradient.npz", d / "warp_gradient.npz")
    shutil.copyfile(res / "warp/gradient20/result.json", d / "warp_result.json")
    with np.load(res / "gradient20_highest_exact/gradients.npz") as g:
        np.savez_compressed(d / "fdtdx_gradient.npz", g0=g["g0"])

    listing = {
        str(p.relative_to(HERE)): p.stat().st_size
        for p in sorted(HERE.rglob("*"))
        if p.is_file() and p.suffix in (".npz", ".json") and p.name != "index.json"
    }
    (HERE / "index.json").write_text(json.dumps(listing, indent=1) + "\n")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <warp-fdtd checkout>")
    main(sys.argv[1])
