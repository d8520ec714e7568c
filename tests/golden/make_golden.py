"""Regenerate the golden fixtures in this folder from the reference's committed run data.

The reference (bniehoff/lennard-jonesium) ships one complete seeded run in
``notebooks/quick_single_run/data``: N=500, rho=0.8, T=0.5, rc=2.5, dt=0.005,
seed 117208264 (``run.ini``).  Its CSVs were written by fmt's ``{}`` format,
which prints the shortest representation that round-trips, so every double
parsed here is bit-identical to the value the reference held in memory.

This script reads those files (it needs the reference checkout, so it only
runs where that checkout exists) and writes:

  quick_single_run.npz
      snapshot_xvf   (500, 9) float64  x, v, F of every atom at step 1600
      thermo_head    (200, 8) float64  rows 0..199 of thermodynamics.csv
      thermo_tail    (1, 8)   float64  the last row (step 1599, the snapshot's state)
      thermo_te      (1600,)  float64  the total-energy column (drift reference)
      observations   (20, 7)  float64  observations.csv
  quick_single_run_run.ini     copy of run.ini
  quick_single_run_events.log  copy of events.log

Usage:  python tests/golden/make_golden.py REFERENCE_ROOT

REFERENCE_ROOT is the directory of a checkout of the reference repository.
"""

import csv
import pathlib
import shutil
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent


def _rows(path, skip):
    with open(path, newline="") as fh:
        rows = list(csv.reader(fh))
    return [[float(v) for v in r] for r in rows[skip:] if r]


def main(ref_root):
    data = pathlib.Path(ref_root) / "notebooks" / "quick_single_run" / "data"
    snap = np.array(_rows(data / "snapshots.csv", 2))  # two header rows
    assert snap.shape == (500, 11) and np.all(snap[:, 0] == 1600)
    assert np.all(snap[:, 1] == np.arange(500))
    thermo = np.array(_rows(data / "thermodynamics.csv", 1))
    assert thermo.shape == (1600, 8)
    obs = np.array(_rows(data / "observations.csv", 1))
    np.savez_compressed(
        HERE / "quick_single_run.npz",
        snapshot_xvf=snap[:, 2:],
        thermo_head=thermo[:200],
        thermo_tail=thermo[-1:],
        thermo_te=thermo[:, 4].copy(),
        observations=obs,
    )
    shutil.copyfile(data / "run.ini", HERE / "quick_single_run_run.ini")
    shutil.copyfile(data / "events.log", HERE / "quick_single_run_events.log")
    print("wrote", HERE / "quick_single_run.npz")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(__doc__)
    main(sys.argv[1])
