"""Regenerate tests/golden/known_answers.json.

Runs the reference's own sequential programs (built from the reference sources
into oracle/_ref/ by `make -C oracle`) and records their answers, together with
the published known-answer values of the C++ standard generators.  Only needs
to run where the reference sources are present; the JSON it writes is
committed and is what the tests read.
"""
import hashlib
import json
import os
import re
import struct
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.path.join(ROOT, "oracle", "_ref")


def run(prog, *args):
    out = subprocess.run([os.path.join(REF, prog)] + [str(a) for a in args], capture_output=True, text=True,
                         check=True).stdout
    return out


def std_mt19937(seed, n):
    # reference keys come from std::mt19937; use the C++ library itself
    src = r'''
#include <random>
#include <cstdio>
#include <cstdlib>
int main(int c, char** v){ std::mt19937 r(strtoul(v[1],0,10)); long n=atol(v[2]);
 for(long i=0;i<n;++i){ unsigned x=r(); fwrite(&x,4,1,stdout);} }
'''
    with tempfile.TemporaryDirectory() as d:
        cpp = os.path.join(d, "g.cpp")
        exe = os.path.join(d, "g")
        open(cpp, "w").write(src)
        subprocess.run(["g++", "-O2", "-o", exe, cpp], check=True)
        raw = subprocess.run([exe, str(seed), str(n)], capture_output=True, check=True).stdout
    return np.frombuffer(raw, dtype=np.uint32).astype(np.int32)


def main():
    if not os.path.exists(os.path.join(REF, "seq_fib")):
        sys.exit("oracle/_ref is not built (make -C oracle with the reference sources present)")
    fib = {}
    for n in list(range(0, 31)) + [34]:
        m = re.search(r"Fibonacci of (\d+) is (-?\d+)", run("seq_fib", n))
        fib[str(n)] = int(m.group(2))
    nq = {}
    for n in range(1, 14):
        m = re.search(r"N-Queens\((\d+)\) = (\d+)", run("seq_nq", n))
        nq[str(n)] = int(m.group(2))
    # reference cilksort / mergesort on gen_vector-format files (size_t n + int32[n])
    sorts = {}
    for n in (1 << 10, 1 << 16, 1 << 20):
        keys = std_mt19937(42, n)
        with tempfile.NamedTemporaryFile(suffix=".bin", delete=False) as f:
            f.write(struct.pack("<Q", n))
            f.write(keys.tobytes())
            path = f.name
        ok_c = "Correct" in run("seq_cilksort", path)
        ok_m = "Correct" in run("seq_mergesort", path)
        os.unlink(path)
        srt = np.sort(keys, kind="stable")
        sorts[str(n)] = {
            "keys_first8": [int(x) for x in keys[:8]],
            "keys_sha256": hashlib.sha256(keys.tobytes()).hexdigest(),
            "sorted_sha256": hashlib.sha256(srt.tobytes()).hexdigest(),
            "reference_seq_cilksort_correct": ok_c,
            "reference_seq_mergesort_correct": ok_m,
        }
    out = {
        "source": "reference sequential programs (evaluation/2-comparison/{fib/seq_fib.c,nq/seq_nq.c,"
                  "cilksort/seq_cilksort.cpp,mergesort/seq_mergesort.cpp}) compiled by oracle/Makefile; "
                  "keys from the C++ standard library std::mt19937",
        "fib": fib,
        "nq": nq,
        "mt19937_seed5489_10000th": 4123659995,
        "mt19937_64_seed5489_10000th": 9981545732273789042,
        "sorts_seed42": sorts,
        "fib_tasks": {"30_0": 2692537, "34_12": 150049},
        "fib_executions": {"30_0": 4038805},
        "nq_tasks": {"13_12": 4674890},
    }
    with open(os.path.join(HERE, "known_answers.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print("wrote", os.path.join(HERE, "known_answers.json"))


if __name__ == "__main__":
    main()
