"""Check served results against the CPU oracle by hash.

bench.py --serve-sample N --serve-hashes FILE writes the SHA-256 of the final
U of N seeded-random requests of the served stream (strict arithmetic).  This
script reruns each of those requests on the CPU oracle to its t_end and
compares the hash of the oracle's final U (and the step count): identical
hashes mean identical results, i.e. relative L1 = 0.

    python tests/served_check.py FILE [--threads T]
"""
import argparse
import hashlib
import json
import os
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))

import numpy as np  # noqa: E402

import oracle  # noqa: E402
import pkg  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("hashes")
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    args = ap.parse_args()
    rec = json.load(open(args.hashes))
    pkg.load()
    import importlib
    problems = importlib.import_module("hosono_2dmhd_b200.problems")
    manifest = os.path.join(pkg.PKG_DIR, "workloads", rec["manifest"])
    entries = {str(e["id"]): e for e in json.load(open(manifest))["requests"]}
    oracle.set_threads(args.threads)
    same = 0
    out = []
    with tempfile.TemporaryDirectory() as d:
        for rid, r in sorted(rec["requests"].items(), key=lambda kv: kv[1]["zone_updates"]):
            e = entries[rid]
            par = problems.make(d, f"r{rid}", problems.from_entry(e))
            t0 = time.time()
            o = oracle.Oracle(par)
            rc, t, n = o.run()
            h = hashlib.sha256(np.ascontiguousarray(o.U()).tobytes()).hexdigest()
            o.close()
            ok = h == r["sha256"] and n == r["nstep"]
            same += ok
            out.append(dict(id=int(rid), problem=e["problem"], n=e["n"], radius=e["radius"], steps=n,
                            identical=ok, cpu_s=round(time.time() - t0, 1)))
            print(json.dumps(out[-1]), flush=True)
    print(json.dumps({"checked": len(out), "identical": same}))
    return 0 if same == len(out) else 1


if __name__ == "__main__":
    sys.exit(main())
