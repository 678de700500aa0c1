"""Generates tests/golden/reference_anchors.json: the reference's published
results for the uniform solver, with the command lines that produced them,
and this implementation's FP64 output for the same commands.

Published (reference, read as text):
  README.md:44, 190, 408-409  Ra = 1e8, 128 x 511, --nu 0.001 --alpha-mult 1.2,
                              2 000 000 steps -> Nuc = 30.45
  README.md:50                y+ of the first cell at Ra = 1e8: 0.63
  README.md:313-318           "curseur DNS/LES": Ra = 1e8, 64 x 256, 1 000 000
                              steps, the same nu, Cs = 0.1 -> Nuc 30.58,
                              nu_t/nu 4.8 %; Cs = 0.2 -> Nuc 29.47, 18.4 %
The cursor runs' sampling follows the README's Ra = 1e8 command (README.md
143-147: --sample-start 300000); their nu is the 128 x 511 run's (0.001,
--alpha-mult 1.2: with --alpha-mult 1.0, tau_t < 0.505 and the solver refuses
the run, as the reference's assert at src/uniform/solver.rs:154 does).

The measured values come from the driver binary (cfd_cavity_b200/_build/
cavity_les, FP64 storage, bit-identical to the FP64 oracle) on a B200:
  python tests/golden/make_anchor_fixture.py      (needs a GPU, ~1 min)
"""
from __future__ import annotations

import json
import os
import re
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
DRIVER = os.path.join(ROOT, "cfd_cavity_b200", "_build", "cavity_les")
OUT = os.path.join(HERE, "reference_anchors.json")

RUNS = {
    "ra1e8_128x511": dict(
        cite="README.md:44, 50, 190, 408-409",
        args=["--nx", "128", "--ny", "511", "--ra", "1e8", "--nu", "0.001", "--alpha-mult", "1.2",
              "--steps", "2000000"],
        published={"nuc": 30.45, "y_plus_hot": 0.63},
        late_window_from=1_500_000),
    "cursor_cs0.1": dict(
        cite="README.md:313-317",
        args=["--nx", "64", "--ny", "256", "--ra", "1e8", "--cs", "0.1", "--nu", "0.001", "--alpha-mult", "1.2",
              "--steps", "1000000", "--sample-start", "300000", "--progress-every", "50000"],
        published={"nuc": 30.58, "nu_t_over_nu_pct": 4.8}),
    "cursor_cs0.2": dict(
        cite="README.md:313-318",
        args=["--nx", "64", "--ny", "256", "--ra", "1e8", "--cs", "0.2", "--nu", "0.001", "--alpha-mult", "1.2",
              "--steps", "1000000", "--sample-start", "300000", "--progress-every", "50000"],
        published={"nuc": 29.47, "nu_t_over_nu_pct": 18.4}),
}
PROGRESS = re.compile(r"step\s+(\d+) \|.*Nuc = ([\d.]+) \| Nuf = ([\d.]+) .*nu_t_max = ([\d.e+-]+)")


def run(name, spec, workdir):
    """Runs the driver; returns the measured quantities."""
    out = os.path.join(workdir, name)
    r = subprocess.run([DRIVER, *spec["args"], "--out", out], capture_output=True, text=True, timeout=900)
    if r.returncode != 0:
        raise RuntimeError(f"{name}: driver exit {r.returncode}\n{r.stderr[-2000:]}")
    rows = [(int(m.group(1)), float(m.group(2)), float(m.group(4)))
            for m in (PROGRESS.match(line) for line in r.stdout.splitlines()) if m]
    with open(os.path.join(out, "summary.json")) as fh:
        summ = json.load(fh)
    nu = 0.001
    meas = {"nuc_mean_field": summ["nusselt_hot"], "nuf_mean_field": summ["nusselt_cold"],
            "y_plus_hot": summ["y_plus_hot"], "nuc_final": rows[-1][1],
            "nu_t_over_nu_pct_final": 100.0 * rows[-1][2] / nu}
    if "late_window_from" in spec:
        sel = [nuc for s, nuc, _ in rows if s >= spec["late_window_from"]]
        meas["nuc_mean_late"] = sum(sel) / len(sel)
    return meas


def main():
    res = {"about": __doc__.split("\n\n")[0], "runs": {}}
    with tempfile.TemporaryDirectory() as wd:
        for name, spec in RUNS.items():
            res["runs"][name] = {**{k: v for k, v in spec.items()}, "measured": run(name, spec, wd)}
            print(name, res["runs"][name]["measured"], flush=True)
    with open(OUT, "w") as fh:
        json.dump(res, fh, indent=1)


if __name__ == "__main__":
    sys.exit(main())
