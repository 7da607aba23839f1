"""Regenerate the golden fixtures of this directory from a gample checkout.

Usage: python tests/golden/make_golden.py /path/to/gample

Copies, unmodified:
  * condition files of the reference (data/*.json) used by the parser and
    physics tests;
  * the reference's recorded timeseries of data/single_darwin.json and
    data/uniform_darwin.json (single_darwin_test_timeseries.csv,
    uniform_darwin_test_timeseries.csv at the repository root), which pin the
    loader, deposit, Poisson solve and phi/E reconstruction;
  * the first 50 logged rows of org_3rd_20250930132346_timeseries.csv, the
    recorded run of data/org_3rd.json (org_3rd_head_timeseries.csv).
"""
import os
import shutil
import sys

CONDITIONS = ["single_darwin", "uniform_darwin", "single", "debye", "periodic", "harmonic",
              "harmonic_sinusoidal", "check_quiet", "org", "org_3rd", "org_5th", "condition_uniform",
              "injection"]
TRACES = ["single_darwin_test_timeseries.csv", "uniform_darwin_test_timeseries.csv"]


# A long recorded run whose first logged rows (every 20 cycles) are kept:
# data/org_3rd.json, 3rd order, 500 x 200, Dirichlet 200 V / 0 V.
HEAD_TRACES = {"org_3rd_20250930132346_timeseries.csv": ("org_3rd_head_timeseries.csv", 50)}


def main(src):
    here = os.path.dirname(os.path.abspath(__file__))
    for name in CONDITIONS:
        shutil.copyfile(os.path.join(src, "data", name + ".json"), os.path.join(here, name + ".json"))
    for t in TRACES:
        shutil.copyfile(os.path.join(src, t), os.path.join(here, t))
    for t, (out, rows) in HEAD_TRACES.items():
        with open(os.path.join(src, t)) as f, open(os.path.join(here, out), "w") as g:
            for k, line in enumerate(f):
                if k > rows:
                    break
                g.write(line)
    print("wrote", len(CONDITIONS), "conditions,", len(TRACES), "traces and", len(HEAD_TRACES), "trace heads to", here)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py /path/to/gample")
    main(sys.argv[1])
