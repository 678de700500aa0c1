"""Generates the golden fixtures of tests/golden/ from the FP64 oracle.

The reference (Rust) cannot be built here, so the fixtures are outputs of the
oracle (oracle/, a restatement of src/uniform/solver.rs and post.rs) on the
benchmark configurations, at sizes too long to rerun inside a test:

  c1_64x256_ra1e6.json   64x256, Ra=1e6, FP64, theta = 0 + U(+-1e-4) (seed 42),
                         20 000 steps;
  c2_128x512_ra1e8.json  128x512, Ra=1e8, same physics, 200 000 steps, Nu
                         averaged over steps 150 001-200 000.

Each run records the final diagnostics, the per-step mean of the
instantaneous Nusselt numbers over the averaging window, the reference's own
estimator (Nusselt of the time-mean temperature sampled every 100 steps,
src/main.rs:279-281, 317-322, 740-753) and a sparse fingerprint of the final
temperature field.

Usage:  python tests/golden/make_golden.py [c1|c2 ...] [--jobs 8]
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))

from oracle import INIT_ZERO, OracleAverager, OracleSolver  # noqa: E402

CONFIGS = {
    "c1": dict(name="c1_64x256_ra1e6", nx=64, ny=256, ra=1e6, steps=20_000, window=5_000),
    "c2": dict(name="c2_128x512_ra1e8", nx=128, ny=512, ra=1e8, steps=200_000, window=50_000),
}
PHYS = dict(pr=0.71, cs=0.10, pr_t=0.9, utarget=0.02, seed=42)
SAMPLE_EVERY = 100
FINGERPRINT_STRIDE = 97


def run(cfg, jobs):
    nx, ny, steps, window = cfg["nx"], cfg["ny"], cfg["steps"], cfg["window"]
    s = OracleSolver(nx, ny, cfg["ra"], PHYS["pr"], PHYS["cs"], PHYS["pr_t"], PHYS["utarget"],
                     PHYS["seed"], jobs, init_mode=INIT_ZERO, noise_amp=1e-4)
    avg = OracleAverager(nx * ny)
    sample_start = steps - window  # 0-based loop index of the first sampled state
    t0 = time.time()
    s.step(sample_start)
    nu_h = nu_c = 0.0
    for step in range(sample_start, steps):
        s.step(1)
        h, c = s.nusselt()
        nu_h += h
        nu_c += c
        if (step - sample_start) % SAMPLE_EVERY == 0:
            avg.accumulate(s)
    elapsed = time.time() - t0
    n_samples, means = avg.means()
    t_mean = means[2]
    d = s.diag()
    t = s.fields()["temperature"]
    out = dict(
        config=dict(nx=nx, ny=ny, ra=cfg["ra"], steps=steps, window=window, init="zero",
                    noise_amp=1e-4, sample_every=SAMPLE_EVERY, **PHYS),
        info=s.info(),
        final=d,
        nu_hot_step_mean=nu_h / window,
        nu_cold_step_mean=nu_c / window,
        nu_hot_of_mean_t=s.nusselt_from_mean(t_mean, True),
        nu_cold_of_mean_t=s.nusselt_from_mean(t_mean, False),
        n_samples=n_samples,
        fingerprint_stride=FINGERPRINT_STRIDE,
        t_fingerprint=t[::FINGERPRINT_STRIDE].tolist(),
        oracle_seconds=elapsed,
        oracle_jobs=jobs,
    )
    path = os.path.join(HERE, cfg["name"] + ".json")
    with open(path, "w") as fh:
        json.dump(out, fh, indent=1)
    print(f"{cfg['name']}: {elapsed:.1f} s, Nu_hot(step mean) {out['nu_hot_step_mean']:.6f}, "
          f"Nu_hot(mean T) {out['nu_hot_of_mean_t']:.6f} -> {path}", flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("which", nargs="*", default=["c1"])
    ap.add_argument("--jobs", type=int, default=os.cpu_count() or 1)
    a = ap.parse_args()
    for w in a.which:
        run(CONFIGS[w], a.jobs)


if __name__ == "__main__":
    main()
