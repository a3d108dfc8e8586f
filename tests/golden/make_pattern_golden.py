"""Oracle counts of P1..P8 on the pattern benchmark graph.

The graph is the seeded Chung-Lu graph bench.py --mode patterns counts by
default (n 100,000, gamma 2.1, mean degree 10, weight cap 200, seed 1), built
by the oracle's own generator restatement.  Every count comes from the CPU
restatement of the reference's formulas (oracle/patterns_oracle.cpp), all
host threads.  The result goes to tests/golden/pattern_counts.json under the
key bench.py uses; tests/test_patterns_gpu.py and bench.py check the GPU
counts against it.

  python tests/golden/make_pattern_golden.py [--n 100000 --mean 10 --cap 200]

With --fast, P1 and P4 come from the second restatement
(oracle/patterns_fast.cpp) and P7 and P8 from their clique restatement
(oracle/clique_patterns.cpp), both pinned to the literal one by
tests/test_oracle.py, which count graphs with hubs in minutes; the Chung-Lu
graph with n 1,000,000, mean 20 and cap 50,000 is counted that way:

  python tests/golden/make_pattern_golden.py --n 1000000 --mean 20 --cap 50000 \
      --patterns 1,4,7,8 --fast

The same shape at 5,000 vertices (hubs of degree 2,187, 1,525 and 1,173)
is small enough for the literal restatement, all eight patterns (P3, whose
correction is quartic in a hub's degree, last; a few minutes on 8 threads):

  python tests/golden/make_pattern_golden.py --n 5000 --mean 20 --cap 50000 \
      --patterns 1,2,4,5,6,7,8,3
"""
import argparse
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
OUT = os.path.join(HERE, "pattern_counts.json")


def key(n, mean, cap):
    return f"chung_lu_n{n}_mean{mean:g}_cap{cap:g}_seed1"


def main():
    from oracle import oracle as orc
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=100000)
    ap.add_argument("--mean", type=float, default=10.0)
    ap.add_argument("--cap", type=float, default=200.0)
    ap.add_argument("--patterns", default="1,2,3,4,5,6,7,8")
    ap.add_argument("--fast", action="store_true",
                    help="P1/P4 by patterns_fast.cpp, P7/P8 by clique_patterns.cpp")
    a = ap.parse_args()
    rp, col = orc.chung_lu(a.n, 2.1, a.mean, a.cap, seed=1)
    rec = json.load(open(OUT)) if os.path.exists(OUT) else {}
    entry = rec.setdefault(key(a.n, a.mean, a.cap), {})
    entry.update({"n": a.n, "m": int(len(col) // 2), "max_degree": int((rp[1:] - rp[:-1]).max()),
                  "source": ("oracle/patterns_fast.cpp (P1, P4) and oracle/clique_patterns.cpp (P7, P8)"
                             if a.fast else "oracle/patterns_oracle.cpp") +
                            " on the oracle's generator restatement"})
    counts = entry.setdefault("counts", {})
    seconds = entry.setdefault("oracle_seconds", {})
    for k in [int(x) for x in a.patterns.split(",") if x]:
        t0 = time.time()
        if not a.fast:
            counts[f"P{k}"] = orc.pattern(rp, col, k)
        elif k in (7, 8):
            counts[f"P{k}"] = orc.clique_patterns(rp, col)[k]
        else:
            counts[f"P{k}"] = orc.pattern_fast(rp, col, k)
        seconds[f"P{k}"] = round(time.time() - t0, 1)
        print(f"P{k}", counts[f"P{k}"], seconds[f"P{k}"], flush=True)
        with open(OUT, "w") as f:
            json.dump(rec, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
