"""Extract the reference's golden vectors for the Omniscape path into small fixtures.

Run in a checkout that has the reference sources (``--ref`` points at the
landschaft source tree).  Reads the reference's own test data:

* ``tests/data/reference/circuit/omniscape.npz``: 8 Omniscape.jl 0.7 runs
  (inputs, options and the CHOLMOD outputs; the cg+amg outputs are left out);
* ``tests/data/reference/circuit/advanced.npz`` + ``advanced_inputs.npz``: 6
  Circuitscape advanced-mode solves (CHOLMOD node currents);
* ``tests/data/reference/circuit/omniscape_ini/*.ini``, ``omniscape_input/*``
  (ASCII grids and a reclass table) and ``omniscape_ini.npz``: 11 Omniscape.jl
  INI runs (the CHOLMOD outputs; the cg+amg outputs are left out);
* ``tests/data/reference/circuit/circuitscape/input/raster/pairwise/*`` and the
  ``sgVerify*`` entries of ``circuitscape.npz``: Circuitscape's 17 pairwise INI
  cases (resistance matrices and current / voltage maps);
* ``.../input/raster/{advanced,one_to_all,all_to_one}/*`` and the ``mgVerify*``,
  ``ex_advanced``, ``oneToAllVerify*`` and ``allToOneVerify*`` entries: the
  advanced, one-to-all and all-to-one INI cases.

Writes ``omniscape_golden.npz``, ``advanced_golden.npz``, ``omniscape_ini.npz``,
``circuitscape/pairwise.npz``, ``circuitscape/modes.npz`` and copies of the INI and input files (same
layout) next to this file.
The GPU machines do not have the reference tree, so the tests read only these
fixtures.
"""

from __future__ import annotations

import argparse
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    args = ap.parse_args()
    data = Path(args.ref) / "tests" / "data" / "reference" / "circuit"
    z = np.load(data / "omniscape.npz")
    out = {}
    for k in z.files:
        if "/cgamg/" in k:
            continue
        out[k] = z[k]
    np.savez_compressed(HERE / "omniscape_golden.npz", **out)
    inp = np.load(data / "advanced_inputs.npz")
    ref = np.load(data / "advanced.npz")
    out = {k: inp[k] for k in inp.files}
    out.update({k: ref[k] for k in ref.files if k.endswith("current_cholmod")})
    np.savez_compressed(HERE / "advanced_golden.npz", **out)
    z = np.load(data / "omniscape_ini.npz")
    np.savez_compressed(HERE / "omniscape_ini.npz", **{k: z[k] for k in z.files if "/cgamg/" not in k})
    for sub in ("omniscape_ini", "omniscape_input"):
        (HERE / sub).mkdir(exist_ok=True)
        for f in sorted((data / sub).iterdir()):
            (HERE / sub / f.name).write_bytes(f.read_bytes())
    cs = data / "circuitscape"
    z = np.load(data / "circuitscape.npz")
    out_dir = HERE / "circuitscape"
    out_dir.mkdir(exist_ok=True)
    np.savez_compressed(out_dir / "pairwise.npz", **{k: z[k] for k in z.files if k.startswith("sgVerify")})
    np.savez_compressed(out_dir / "modes.npz", **{k: z[k] for k in z.files
                                                 if k.startswith(("mgVerify", "ex_advanced", "oneToAll", "allToOne"))})
    sub = ("pairwise", "advanced", "one_to_all", "all_to_one")
    for f in sorted(x for s in sub for x in (cs / "input" / "raster" / s).rglob("*")):
        if f.is_file():
            dst = out_dir / f.relative_to(cs)
            dst.parent.mkdir(parents=True, exist_ok=True)
            dst.write_bytes(f.read_bytes())


if __name__ == "__main__":
    main()
