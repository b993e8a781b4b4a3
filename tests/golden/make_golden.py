"""Regenerates the golden fixtures in this folder from the reference tree.

The fixtures are outputs the reference itself committed (it cannot be run
here: Julia is not installed).  This script only copies and subsets them:

* tdvp_benchmark.csv   <- tdvp_benchmark_results.csv (test/benchmark_tdvp.jl:94-216):
                          L=6, dt=0.05, T=2, <Z> at sites 1,3,6; Exact, 1TDVP and 2TDVP rows.
* large_ising.csv      <- large_ising_results.csv (test/simulate_large_ising.jl:31-98):
                          L=30 Ising 2TDVP, chi<=32, <Z> at sites 1,16,30.
* tjm_vs_qutip_a.csv,
  tjm_vs_qutip_b.csv   <- 00_safety_checks_full_algorithms/analogTJM_check/{,non_long_range_check/}
                          results/tjm_vs_qutip_data.csv (benchmark_analog_tjm.jl:90-227):
                          columns t, TJM <Z_1..6>, TJM stagg, QuTiP <Z_1..6>, QuTiP stagg.

Usage: python tests/golden/make_golden.py /path/to/reference
"""
import csv
import os
import shutil
import sys

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("YAQS_REFERENCE_TREE")
if not REF:
    sys.exit(f"usage: python {os.path.basename(__file__)} /path/to/reference  (or set YAQS_REFERENCE_TREE)")
HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    with open(os.path.join(REF, "tdvp_benchmark_results.csv")) as f, \
            open(os.path.join(HERE, "tdvp_benchmark.csv"), "w", newline="") as g:
        r = csv.reader(f)
        w = csv.writer(g)
        w.writerow(next(r))
        for row in r:
            if row[1] in ("Exact", "1TDVP", "2TDVP"):
                w.writerow(row)
    shutil.copyfile(os.path.join(REF, "large_ising_results.csv"), os.path.join(HERE, "large_ising.csv"))
    base = os.path.join(REF, "00_safety_checks_full_algorithms", "analogTJM_check")
    shutil.copyfile(os.path.join(base, "results", "tjm_vs_qutip_data.csv"),
                    os.path.join(HERE, "tjm_vs_qutip_a.csv"))
    shutil.copyfile(os.path.join(base, "non_long_range_check", "results", "tjm_vs_qutip_data.csv"),
                    os.path.join(HERE, "tjm_vs_qutip_b.csv"))


if __name__ == "__main__":
    main()
