"""Regenerate the function golden vectors from sundog's own device headers.

Runs oracle/_ref/fnvec_ref (oracle/fnvec.cpp compiled against the reference
device/*.cuh by `make -C oracle ref`) on seeded inputs from oracle/items.py
and stores inputs and outputs as tests/golden/fnvec_<name>.npz. Needs the
reference sources (this script is not run by the tests).

    python tests/golden/make_golden.py
"""

import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import items  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref", "fnvec_ref")
COUNTS = {1: 256, 2: 4096, 3: 4096, 4: 4096, 6: 4096, 7: 512, 8: 2048, 9: 2048}
SEEDS = {1: 101, 2: 102, 3: 103, 4: 104, 6: 106, 7: 107, 8: 108, 9: 109}


def run_ref(which, payload, n, out_dtype):
    with tempfile.TemporaryDirectory() as d:
        fi, fo = os.path.join(d, "in.bin"), os.path.join(d, "out.bin")
        with open(fi, "wb") as f:
            f.write(payload)
        subprocess.run([REF, str(which), str(n), fi, fo, str(out_dtype.itemsize)], check=True)
        return np.fromfile(fo, out_dtype)


def main():
    if not os.path.isfile(REF):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True)
    for which, n in COUNTS.items():
        name, din, dout = items.ITEMS[which]
        a = items.generate(which, n, SEEDS[which])
        extra = b""
        if which == 9:
            table = items.cdf_table(SEEDS[which])
            # Probe exactly on entries too: the search's tie rule.
            a["u"][: len(table) - 1] = table[:-1]
            extra = np.int32(len(table)).tobytes() + table.tobytes()
        payload = a.tobytes() + extra
        out = run_ref(which, payload, n, dout)
        path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "fnvec_%s.npz" % name)
        np.savez_compressed(path, which=which, input=np.frombuffer(payload, np.uint8),
                            output=np.frombuffer(out.tobytes(), np.uint8), n=n)
        print("wrote", path, n, "items")


if __name__ == "__main__":
    main()
