"""Regenerates tests/golden/*.csv: the reference's regression statistics (golden vectors) for the
cases on this path, reduced to the columns the reference's own
comparison uses (tests/regression/compare_stats.py: time, E, Umax, Ub, tauw_mean, nu_sgs_mean,
max_abs_divU), plus the dissipation and the cell-velocity divergence columns.  Run in a checkout that has the reference tree:

    python tests/golden/make_golden.py /path/to/reference
"""
import csv
import os
import sys

CASES = ("tgv", "tgv_skew", "tgv_skew_chk", "pdrop", "hydro", "hydrowall", "rb", "channel", "amd", "graded",
         "channel_most", "duct", "duct_exact", "hydro_exact", "tgv_skew_exact", "default_skew", "inflow",
         "inflow_jarrin")
COLS = ("step", "time", "E", "eps", "Umax", "Ub", "tauw_mean", "nu_sgs_mean", "max_abs_divU", "max_abs_divU_cell",
        "volavg_abs_divU_cell", "dt")


def main(ref_root):
    here = os.path.dirname(os.path.abspath(__file__))
    for case in CASES:
        src = os.path.join(ref_root, "tests", "regression", "reference", f"{case}_np1.csv")
        with open(src, newline="") as fh:
            rows = list(csv.DictReader(fh))
        dst = os.path.join(here, f"{case}_np1.csv")
        with open(dst, "w", newline="") as fh:
            w = csv.writer(fh)
            w.writerow(COLS)
            for r in rows:
                w.writerow([r[c].strip() for c in COLS])
        print(f"{dst}: {len(rows)} rows")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path to the reference checkout>")
    main(sys.argv[1])
