"""Regenerate the golden fixtures of this directory from a gample checkout.

Usage: python tests/golden/make_golden.py /path/to/gample

Copies, unmodified:
  * condition files of the reference (data/*.json) used by the parser and
    physics tests;
  * the reference's recorded timeseries of data/single_darwin.json and
    data/uniform_darwin.json (single_darwin_test_timeseries.csv,
    uniform_darwin_test_timeseries.csv at the repository root), which pin the
    loader, deposit, Poisson solve and phi/E reconstruction.
"""
import os
import shutil
import sys

CONDITIONS = ["single_darwin", "uniform_darwin", "single", "debye", "periodic", "harmonic",
              "harmonic_sinusoidal", "check_quiet", "org", "org_3rd", "org_5th", "condition_uniform",
              "injection"]
TRACES = ["single_darwin_test_timeseries.csv", "uniform_darwin_test_timeseries.csv"]


def main(src):
    here = os.path.dirname(os.path.abspath(__file__))
    for name in CONDITIONS:
        shutil.copyfile(os.path.join(src, "data", name + ".json"), os.path.join(here, name + ".json"))
    for t in TRACES:
        shutil.copyfile(os.path.join(src, t), os.path.join(here, t))
    print("wrote", len(CONDITIONS), "conditions and", len(TRACES), "traces to", here)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py /path/to/gample")
    main(sys.argv[1])
