"""Effective-tensor columns of the golden cases computed by the oracle, for the GPU parity
tests (which run where the oracle's CPU solve of these 1-3 M DOF cases would be slow).

The oracle is the reference's own host code driving the CPU restatement of its solver
(oracle/_ref/chfem_oracle_exec, built by `make -C oracle ref`).  Each entry records the
settings it was run with.  Usage: python tests/golden/make_oracle_columns.py
"""
import json
import os
import sys
import tempfile

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))
from tests import helpers as H  # noqa: E402

RUNS = [
    # key, golden case, extra CLI flags
    ("thermal_x_pcg", "thermal_ggg40", ["-d", "0"]),
    ("elastic_y_pcg", "elastic_ggg40", ["-d", "1"]),
    ("fluid_z_pcg", "fluid_fibers", ["-d", "2"]),
    ("fluid_z_pminres", "fluid_fibers", ["-d", "2", "-s", "1"]),
    ("thermal_all_pcg", "thermal_ggg40", []),
]


def main():
    out = {}
    with tempfile.TemporaryDirectory() as wd:
        for key, case, flags in RUNS:
            nf, raw, meta = H.golden_case_files(case, wd)
            C, log = H.run_exec(H.ORACLE_EXEC, nf, raw, *flags, env={"OMP_NUM_THREADS": str(os.cpu_count() or 4)})
            its = H.parse_iterations(log)
            out[key] = {"case": case, "flags": flags, "C": C.tolist(), "iterations": its}
            print(key, its, flush=True)
    with open(os.path.join(H.GOLDEN, "oracle_columns.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
