"""Times the CPU restatement on a bounded sample of the bench workload
(TEST INFRASTRUCTURE: the CPU baseline legs of bench.py run it).

    IFC_ORACLE_LIB=oracle/_build/libifc_oracle_omp.so OMP_NUM_THREADS=16 \\
        python oracle/time_port.py --seconds 10 --nx 512 --ny 128

runs outer iterations of the 2D channel from rest (FP32, red-black sweeps)
until the given seconds have passed and prints one JSON line: outer
iterations, relaxed cell-updates, seconds and the threads OpenMP used.
"""
import argparse
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "incompflow-cuda_b200", "python"))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "tests"))

import ifc  # noqa: E402  (configs only; the library is not loaded)
import oracle as O  # noqa: E402
from helpers import to_oracle_cfg  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--seconds", type=float, default=10.0)
    ap.add_argument("--nx", type=int, default=512)
    ap.add_argument("--ny", type=int, default=128)
    a = ap.parse_args()
    o = O.Oracle(to_oracle_cfg(ifc.channel2d(a.nx, a.ny)), "f")
    t0 = time.perf_counter()
    its = updates = 0
    while time.perf_counter() - t0 < a.seconds:
        nm = o.outer_iteration()
        its += 1
        updates += o.N * (nm["sweeps"][0] + nm["sweeps"][1] + nm["sweeps"][3])
    dt = time.perf_counter() - t0
    print(json.dumps({"outer_iterations": its, "cell_updates": updates, "seconds": dt,
                      "threads": int(os.environ.get("OMP_NUM_THREADS", "1")), "lib": os.path.basename(O.LIB_PATH)}))


if __name__ == "__main__":
    main()
